/*
 * CPU oracle for the conjugate-gradient hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's serial CG backend (hahnjo/CGxx),
 * used by tests/, the smoke check and bench.py's CPU-baseline leg as the
 * checker. Nothing in the product links or calls this library.
 *
 * Every function cites the reference file:line it restates. Arithmetic is
 * kept in the reference's order (sequential row sums, sequential dots,
 * separate multiply and add: the library is built with -ffp-contract=off) so
 * that its results are bit-identical to the reference's `cg_serial` built
 * with g++ -O3 on x86-64; tests/test_oracle.py pins that against the
 * reference binaries built by oracle/Makefile into oracle/_ref/ and against
 * the committed fixtures in tests/golden/.
 */
#ifndef CG_ORACLE_H
#define CG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Matrix in coordinate form, rows/cols 0-based (Matrix.h:22-31). */
typedef struct {
  int N;
  int nz;
  int *I;
  int *J;
  double *V;
  int *nzPerRow;
} orc_coo;

/* Status codes of orc_read_mtx; each mirrors one exit(1) path of
 * MatrixCOO::MatrixCOO (Matrix.cpp:13-111). */
enum {
  ORC_OK = 0,
  ORC_ERR_OPEN = 1,         /* "Can't open file with matrix!" */
  ORC_ERR_BANNER = 2,       /* "Only supporting real matrices in coordinate format!" */
  ORC_ERR_STORAGE = 3,      /* "Only supporting general or symmetric matrices!" */
  ORC_ERR_NOT_SQUARE = 4,   /* "Need a square matrix!" */
  ORC_ERR_PARSE = 5,        /* "An exception occurred while reading the matrix!" */
};

int orc_read_mtx(const char *path, orc_coo *out);
void orc_coo_free(orc_coo *c);
int orc_coo_max_nz(const orc_coo *c);

/* COO -> CRS keeping file order inside each row (Matrix.cpp:203-228). */
void orc_coo_to_crs(const orc_coo *c, int *ptr, int *index, double *value);
/* COO -> column-major ELL, k = j*N + i (Matrix.cpp:339-361). Padding slots
 * (j >= length[i]) are left untouched. */
void orc_coo_to_ell(const orc_coo *c, int maxNz, int *length, int *index,
                    double *data);
/* C[i] = 1 / A_ii from the COO diagonal (Preconditioner.cpp:13-23). */
void orc_jacobi_init(const orc_coo *c, double *C);
/* k = A * 1, i.e. row sums in COO order (CG.cpp:256-261). */
void orc_rhs_ones(const orc_coo *c, double *k);

/* Serial kernels (serial/SerialCG.cpp). */
void orc_matvec_coo(int N, int nz, const int *I, const int *J, const double *V,
                    const double *x, double *y);                 /* :79-85  */
void orc_matvec_crs(int N, const int *ptr, const int *index,
                    const double *value, const double *x, double *y); /* :87-95 */
void orc_matvec_ell(int N, const int *length, const int *index,
                    const double *data, const double *x, double *y); /* :97-106 */
void orc_axpy(int N, double a, const double *x, double *y);  /* :127-134 */
void orc_xpay(int N, const double *x, double a, double *y);  /* :136-143 */
double orc_dot(int N, const double *a, const double *b);     /* :145-155 */
void orc_jacobi_apply(int N, const double *C, const double *x,
                      double *y);                            /* :157-161 */

/* Matrix given to the solver: exactly one of the three formats is set. */
enum { ORC_FMT_COO = 0, ORC_FMT_CRS = 1, ORC_FMT_ELL = 2 };
typedef struct {
  int format;
  int N;
  int nz;
  /* COO */
  const int *I, *J;
  const double *V;
  /* CRS */
  const int *ptr, *index;
  const double *value;
  /* ELL (index/data reuse the CRS names) */
  const int *length;
  const double *data;
} orc_matrix;

/* CG::solve (CG.cpp:284-385). x holds x0 on entry and the solution on exit.
 * C == NULL selects PreconditionerNone. Returns the iteration count as
 * CG::printSummary reports it; *residual receives the last relative
 * recurrence residual. */
int orc_cg_solve(const orc_matrix *A, const double *C, const double *k,
                 double *x, int maxIterations, double tolerance,
                 double *residual);

/* CG::check (CG.cpp:387-408): number of |x_i - 1| > checkTolerance. */
int orc_check_ones(int N, const double *x, double checkTolerance);

/* ---------------------------------------------------------------------------
 * Mixed precision (no counterpart in the reference): FP32 Jacobi-PCG inner
 * solves inside an FP64 iterative-refinement loop. The restatement of the
 * scheme that the device solver runs; it is the oracle for its iteration
 * counts and its FP64 true residual.
 *   outer: r = b - A x (FP64); stop when ||r|| / ||b|| <= tolerance;
 *          inner PCG on A d = r in FP32 to relative tolerance innerTol
 *          (FP64 accumulation of dot products); x += d (FP64).
 * Returns total inner iterations; *outer receives outer steps and
 * *trueResidual the final FP64 ||b - A x|| / ||b||. */
int orc_mixed_ir_solve(int N, const int *ptr, const int *index,
                       const double *value, const double *C, const double *b,
                       double *x, int maxIterations, double tolerance,
                       double innerTol, int maxOuter, int *outer,
                       double *trueResidual);

#ifdef __cplusplus
}
#endif

#endif
