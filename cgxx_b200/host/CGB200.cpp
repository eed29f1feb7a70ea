// CGB200: the B200 backend of cg_b200, a CG subclass over libcgb200's C ABI.
// It takes the place of the reference's CUDA plug-in (cuda/CGCUDA.cu,
// cuda/CGCUDABase.h): same supported switches plus COO, device buffers kept
// across repetitions, and the whole solve handed to the device through
// fusedSolve() (one CUDA graph per solve), unless CG_B200_FUSED=0 asks for
// the reference's kernel-by-kernel driving.
//
// Additional environment switches (all optional):
//   CG_B200_FUSED      1 (default) fused device solve, 0 per-kernel calls
//   CG_B200_PRECISION  fp64 (default) | mixed  (FP32 inner + FP64 refinement,
//                      Jacobi)
//   CG_B200_LOOP       graph (default) | chunked | kernels (per-kernel
//                      device times in the summary)
//   CG_B200_DEVICE     CUDA device ordinal (default 0)
//   CG_B200_LEARNED    a weight file of the learned preconditioner (e.g.
//                      cgxx_b200/weights/diffusion7.gnn): M^-1 = G G^T + eps C
//                      with G from the network, inside the mixed-precision
//                      solve (implies CG_B200_PRECISION=mixed; needs Jacobi,
//                      which is also the fallback, and the fused solve). The
//                      factor is built once per upload, like Jacobi::init,
//                      and its time is printed in the summary.
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "CG.h"
#include "cgx.h"

namespace {

[[noreturn]] void fatal() {
  std::cerr << cgx_last_error() << std::endl;
  std::exit(1);
}

void ok(cgx_status s) {
  if (s != CGX_SUCCESS) fatal();
}

[[noreturn]] void badEnv(const char *name, const char *allowed) {
  std::cerr << "Invalid value for " << name << "! (" << allowed << ")"
            << std::endl;
  std::exit(1);
}

// Parameters of a weight file written by cgxx_b200/learned.py: the magic
// "CGXGNN01", a little-endian uint32 header length, a JSON header (not
// needed here) and cgx_gnn_param_count() little-endian floats.
std::vector<float> readWeights(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    std::cerr << "Could not open weight file " << path << "!" << std::endl;
    std::exit(1);
  }
  char magic[8];
  std::uint32_t len = 0;
  const int n = cgx_gnn_param_count();
  std::vector<float> params((size_t)n);
  bool good = (bool)f.read(magic, 8) && std::memcmp(magic, "CGXGNN01", 8) == 0 &&
              (bool)f.read(reinterpret_cast<char *>(&len), 4) &&
              (bool)f.seekg(len, std::ios::cur) &&
              (bool)f.read(reinterpret_cast<char *>(params.data()),
                           (std::streamsize)(sizeof(float) * params.size()));
  if (good) {
    f.peek();
    good = f.eof();  // nothing after the parameters
  }
  if (!good) {
    std::cerr << "Invalid weight file " << path << "! (expected " << n
              << " parameters)" << std::endl;
    std::exit(1);
  }
  return params;
}

}  // namespace

class CGB200 : public CG {
  cgx_handle *h = nullptr;
  bool uploaded = false;
  bool fused = true;
  int precision = CGX_PRECISION_FP64;
  int loop = CGX_LOOP_GRAPH;
  int device = 0;
  cgx_result last{};
  // Learned preconditioner (CG_B200_LEARNED).
  std::string learnedFile;
  std::vector<float> learnedParams;
  cgx_gnn *gnn = nullptr;
  double learnedSetupSeconds = 0;
  static constexpr double kLearnedEps = 1e-4;

  static cgx_vector vec(Vector v) { return (cgx_vector)v; }

  bool supportsMatrixFormat(MatrixFormat) override { return true; }
  bool supportsPreconditioner(Preconditioner p) override {
    return p == PreconditionerJacobi;
  }

  void allocateK() override {
    ok(cgx_host_alloc((void **)&k, sizeof(floatType) * (size_t)N));
  }
  void deallocateK() override {
    cgx_host_free(k);
    k = nullptr;
  }
  void allocateX() override {
    ok(cgx_host_alloc((void **)&x, sizeof(floatType) * (size_t)N));
  }
  void deallocateX() override {
    cgx_host_free(x);
    x = nullptr;
  }

  bool needsTransfer() override { return true; }
  // The COO entries go to the device, which sorts them into CRS or ELL
  // (cgx_upload_coo_as): the same arrays as the host conversion, bit for bit.
  bool convertsOnDevice() override { return true; }

  void doTransferTo() override {
    if (!uploaded) {
      static const int formats[] = {CGX_FORMAT_COO, CGX_FORMAT_CRS, CGX_FORMAT_ELL};
      ok(cgx_upload_coo_as(h, N, nz, matrixCOO->I.get(), matrixCOO->J.get(),
                           matrixCOO->V.get(), formats[matrixFormat]));
      // Later repetitions reuse the device copy; the host COO is not needed.
      if (matrixFormat != MatrixFormatCOO) matrixCOO.reset();
      if (preconditioner == PreconditionerJacobi)
        ok(cgx_upload_jacobi(h, jacobi->C));
      ok(cgx_set_vector(h, CGX_VECTOR_K, k));
      if (gnn) {
        // The learned factor for this matrix: scaled graph and inference.
        const auto t0 = std::chrono::steady_clock::now();
        ok(cgx_learned_setup(h));
        ok(cgx_learned_factor(h, gnn, kLearnedEps));
        ok(cgx_synchronize(h));
        learnedSetupSeconds = std::chrono::duration<double>(
                                  std::chrono::steady_clock::now() - t0)
                                  .count();
      }
      uploaded = true;
    }
    ok(cgx_set_vector(h, CGX_VECTOR_X, x));
    ok(cgx_synchronize(h));
  }

  void doTransferFrom() override { ok(cgx_get_vector(h, CGX_VECTOR_X, x)); }

  void cpy(Vector dst, Vector src) override {
    ok(cgx_copy(h, vec(dst), vec(src)));
  }
  void matvecKernel(Vector xv, Vector yv) override {
    ok(cgx_matvec(h, vec(xv), vec(yv)));
    ok(cgx_synchronize(h));
  }
  void axpyKernel(floatType a, Vector xv, Vector yv) override {
    ok(cgx_axpy(h, a, vec(xv), vec(yv)));
    ok(cgx_synchronize(h));
  }
  void xpayKernel(Vector xv, floatType a, Vector yv) override {
    ok(cgx_xpay(h, vec(xv), a, vec(yv)));
    ok(cgx_synchronize(h));
  }
  floatType vectorDotKernel(Vector a, Vector b) override {
    double r = 0;
    ok(cgx_dot(h, vec(a), vec(b), &r));
    return r;
  }
  void applyPreconditionerKernel(Vector xv, Vector yv) override {
    ok(cgx_apply_jacobi(h, vec(xv), vec(yv)));
    ok(cgx_synchronize(h));
  }

  bool fusedSolve() override {
    if (!fused) return false;
    cgx_options o;
    ok(cgx_default_options(&o));
    o.max_iterations = maxIterations;
    o.tolerance = tolerance;
    o.preconditioner = gnn ? CGX_PRECONDITIONER_LEARNED
                           : preconditioner == PreconditionerJacobi
                               ? CGX_PRECONDITIONER_JACOBI
                               : CGX_PRECONDITIONER_NONE;
    o.precision = precision;
    o.loop = loop;
    ok(cgx_solve(h, &o, &last));
    iteration = last.iterations;
    residual = last.residual;
    if (loop == CGX_LOOP_KERNELS) {
      // Step 1 is the SpMV (+ <p,q>), step 2 the axpy on r (+ dots and the
      // Jacobi apply), step 3 the x and p updates (axpy + xpay).
      setKernelTimes(last.spmv_ms * 1e-3, last.update_ms * 1e-3,
                     last.direction_ms * 1e-3, 0.0, 0.0);
    } else {
      setKernelTimes(last.solve_ms * 1e-3, 0.0, 0.0, 0.0, 0.0);
    }
    return true;
  }

public:
  CGB200() : CG(MatrixFormatCRS, PreconditionerJacobi) {}

  void parseEnvironment() override {
    CG::parseEnvironment();
    if (const char *v = std::getenv("CG_B200_FUSED"); v && *v)
      fused = std::string(v) != "0";
    if (const char *v = std::getenv("CG_B200_PRECISION"); v && *v) {
      std::string s(v);
      if (s == "fp64")
        precision = CGX_PRECISION_FP64;
      else if (s == "mixed")
        precision = CGX_PRECISION_MIXED;
      else
        badEnv("CG_B200_PRECISION", "fp64, or mixed");
      if (precision == CGX_PRECISION_MIXED &&
          preconditioner != PreconditionerJacobi) {
        std::cerr << "Mixed precision needs Jacobi!" << std::endl;
        std::exit(1);
      }
    }
    if (const char *v = std::getenv("CG_B200_LOOP"); v && *v) {
      std::string s(v);
      if (s == "graph")
        loop = CGX_LOOP_GRAPH;
      else if (s == "chunked")
        loop = CGX_LOOP_CHUNKED;
      else if (s == "kernels")
        loop = CGX_LOOP_KERNELS;
      else if (s == "persistent")
        loop = CGX_LOOP_PERSISTENT;
      else if (s == "split")
        loop = CGX_LOOP_PERSISTENT_SPLIT;
      else
        badEnv("CG_B200_LOOP", "graph, chunked, kernels, persistent, or split");
    }
    if (const char *v = std::getenv("CG_B200_DEVICE"); v && *v) {
      char *end = nullptr;
      long d = std::strtol(v, &end, 0);
      if (*end != 0 || d < 0) badEnv("CG_B200_DEVICE", "a device ordinal");
      device = (int)d;
    }
    if (const char *v = std::getenv("CG_B200_LEARNED"); v && *v) {
      const char *pv = std::getenv("CG_B200_PRECISION");
      if (pv && *pv && std::string(pv) != "mixed") {
        std::cerr << "The learned preconditioner runs in mixed precision!"
                  << std::endl;
        std::exit(1);
      }
      if (preconditioner != PreconditionerJacobi || !fused) {
        std::cerr << "The learned preconditioner needs Jacobi and the fused solve!"
                  << std::endl;
        std::exit(1);
      }
      learnedFile = v;
      learnedParams = readWeights(learnedFile);
      precision = CGX_PRECISION_MIXED;
    }
  }

  // The matrix is read first so that file errors are reported before any
  // device error, in the reference's order (CGCUDA::init reads in CG::init).
  void init(const char *matrixFile) override {
    CG::init(matrixFile);
    ok(cgx_create(&h, device));
    if (!learnedParams.empty()) ok(cgx_gnn_create(&gnn, device, learnedParams.data()));
  }

  void printSummary() override {
    CG::printSummary();
    if (fused) {
      std::cout << std::endl;
      printPadded("Device solve time:", std::to_string(last.solve_ms * 1e-3));
      printPadded("Precision:", precision == CGX_PRECISION_MIXED
                                    ? "FP32 inner / FP64 refinement"
                                    : "FP64");
      if (precision == CGX_PRECISION_MIXED) {
        printPadded("Refinement steps:", std::to_string(last.outer_iterations));
        printPadded("Fell back to FP64:", last.fell_back ? "yes" : "no");
        static const char *forms[] = {"per-iteration kernels",
                                      "persistent, fused (band)",
                                      "persistent, split (band)",
                                      "persistent, split (SELL-U)"};
        const int f = last.inner_form >= 0 && last.inner_form <= 3 ? last.inner_form : 0;
        printPadded("Inner solves:", forms[f]);
      }
      if (gnn) {
        printPadded("Learned factor:", learnedFile);
        printPadded("Learned set-up time:", std::to_string(learnedSetupSeconds));
      }
      static const char *loops[] = {"CUDA graph (while node)",
                                    "CUDA graph chunks", "kernel launches",
                                    "persistent inner solves",
                                    "persistent inner solves (split)"};
      printPadded("Device loop:", loops[loop]);
    }
  }

  void cleanup() override {
    CG::cleanup();
    if (gnn) cgx_gnn_destroy(gnn);
    gnn = nullptr;
    if (h) cgx_destroy(h);
    h = nullptr;
  }
};

CG *CG::getInstance() { return new CGB200; }
