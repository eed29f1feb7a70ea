/*
 * CPU oracle for the conjugate-gradient hot path -- TEST INFRASTRUCTURE ONLY.
 * See cg_oracle.h. Built with -O2 -ffp-contract=off so every multiply and add
 * is rounded separately, as in the reference's serial kernels compiled for
 * baseline x86-64 (no FMA).
 */
#include "cg_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* MatrixMarket reader: MatrixCOO::MatrixCOO (Matrix.cpp:13-111).            */

static int read_line(FILE *f, char **buf, size_t *cap) {
  /* getline() semantics of std::getline: strips the '\n'. Returns -1 at EOF
   * with nothing read. */
  ssize_t n = getline(buf, cap, f);
  if (n < 0) return -1;
  if (n > 0 && (*buf)[n - 1] == '\n') (*buf)[--n] = 0;
  return (int)n;
}

static void lower_str(char *s) {
  for (; *s; ++s) *s = (char)tolower((unsigned char)*s);
}

int orc_read_mtx(const char *path, orc_coo *out) {
  memset(out, 0, sizeof(*out));
  FILE *f = fopen(path, "r");
  if (!f) return ORC_ERR_OPEN;
  char *line = NULL;
  size_t cap = 0;
  int rc = ORC_OK;

  /* Banner: five whitespace-separated words, compared case-insensitively
   * except for the first (Matrix.cpp:28-47). */
  char banner[64] = {0}, mtx[64] = {0}, crd[64] = {0}, type[64] = {0},
       storage[64] = {0};
  if (read_line(f, &line, &cap) < 0) line = strdup(""), cap = 1;
  sscanf(line, "%63s %63s %63s %63s %63s", banner, mtx, crd, type, storage);
  lower_str(mtx);
  lower_str(crd);
  lower_str(type);
  lower_str(storage);
  if (strcmp(banner, "%%MatrixMarket") || strcmp(mtx, "matrix") ||
      strcmp(crd, "coordinate") || strcmp(type, "real")) {
    rc = ORC_ERR_BANNER;
    goto done;
  }
  int symmetric = 0;
  if (!strcmp(storage, "symmetric")) {
    symmetric = 1;
  } else if (strcmp(storage, "general")) {
    rc = ORC_ERR_STORAGE;
    goto done;
  }

  /* Skip empty and comment lines (Matrix.cpp:50-53). */
  int n;
  do {
    n = read_line(f, &line, &cap);
    if (n < 0) {
      rc = ORC_ERR_PARSE;
      goto done;
    }
  } while (n == 0 || line[0] == '%');

  int M = 0, N = 0, nz = 0;
  if (sscanf(line, "%d %d %d", &M, &N, &nz) != 3) {
    rc = ORC_ERR_PARSE;
    goto done;
  }
  if (N != M) {
    rc = ORC_ERR_NOT_SQUARE;
    goto done;
  }
  /* Symmetric files store one triangle; the reference sizes the arrays as
   * if every diagonal entry is present (Matrix.cpp:66-69). */
  if (symmetric) nz = 2 * nz - N;

  out->N = N;
  out->nz = nz;
  out->I = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
  out->J = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
  out->V = (double *)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
  out->nzPerRow = (int *)calloc((size_t)(N > 0 ? N : 1), sizeof(int));

  /* Entries: 1-based to 0-based; an off-diagonal entry of a symmetric file
   * is mirrored into the very next slot (Matrix.cpp:80-103). */
  for (int i = 0; i < nz; i++) {
    if (read_line(f, &line, &cap) < 0) {
      rc = ORC_ERR_PARSE;
      goto done;
    }
    char *p = line, *end;
    long r = strtol(p, &end, 10);
    if (end == p) { rc = ORC_ERR_PARSE; goto done; }
    p = end;
    long c = strtol(p, &end, 10);
    if (end == p) { rc = ORC_ERR_PARSE; goto done; }
    p = end;
    double v = strtod(p, &end);
    if (end == p) { rc = ORC_ERR_PARSE; goto done; }
    if (r < 1 || r > N || c < 1 || c > N) { rc = ORC_ERR_PARSE; goto done; }
    out->I[i] = (int)r - 1;
    out->J[i] = (int)c - 1;
    out->V[i] = v;
    out->nzPerRow[out->I[i]]++;
    if (symmetric && out->I[i] != out->J[i]) {
      i++;
      if (i >= nz) { rc = ORC_ERR_PARSE; goto done; }
      out->I[i] = out->J[i - 1];
      out->J[i] = out->I[i - 1];
      out->V[i] = out->V[i - 1];
      out->nzPerRow[out->I[i]]++;
    }
  }

done:
  free(line);
  fclose(f);
  if (rc != ORC_OK) orc_coo_free(out);
  return rc;
}

void orc_coo_free(orc_coo *c) {
  free(c->I);
  free(c->J);
  free(c->V);
  free(c->nzPerRow);
  memset(c, 0, sizeof(*c));
}

/* MatrixCOO::getMaxNz (Matrix.cpp:113-121). */
int orc_coo_max_nz(const orc_coo *c) {
  int m = 0;
  for (int i = 0; i < c->N; i++)
    if (c->nzPerRow[i] > m) m = c->nzPerRow[i];
  return m;
}

/* DataMatrix<MatrixDataCRS>::convert (Matrix.cpp:203-228). */
void orc_coo_to_crs(const orc_coo *c, int *ptr, int *index, double *value) {
  int N = c->N;
  int *offsets = (int *)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  ptr[0] = 0;
  for (int i = 1; i <= N; i++) {
    offsets[i - 1] = ptr[i - 1];
    ptr[i] = ptr[i - 1] + c->nzPerRow[i - 1];
  }
  for (int i = 0; i < c->nz; i++) {
    int row = c->I[i];
    index[offsets[row]] = c->J[i];
    value[offsets[row]] = c->V[i];
    offsets[row]++;
  }
  free(offsets);
}

/* DataMatrix<MatrixDataELL>::convert (Matrix.cpp:339-361); element offsets
 * are 64-bit here so that maxNz * N beyond 2^31 stays defined. */
void orc_coo_to_ell(const orc_coo *c, int maxNz, int *length, int *index,
                    double *data) {
  int N = c->N;
  (void)maxNz;
  memcpy(length, c->nzPerRow, sizeof(int) * (size_t)N);
  int *offsets = (int *)calloc((size_t)(N > 0 ? N : 1), sizeof(int));
  for (int i = 0; i < c->nz; i++) {
    int row = c->I[i];
    size_t k = (size_t)offsets[row] * (size_t)N + (size_t)row;
    index[k] = c->J[i];
    data[k] = c->V[i];
    offsets[row]++;
  }
  free(offsets);
}

/* Jacobi::init (Preconditioner.cpp:13-23): the last diagonal entry in file
 * order wins; rows without one keep whatever C held. */
void orc_jacobi_init(const orc_coo *c, double *C) {
  for (int i = 0; i < c->nz; i++) {
    if (c->I[i] != c->J[i]) continue;
    C[c->I[i]] = 1 / c->V[i];
  }
}

/* CG::init right-hand side (CG.cpp:256-261). */
void orc_rhs_ones(const orc_coo *c, double *k) {
  memset(k, 0, sizeof(double) * (size_t)c->N);
  for (int i = 0; i < c->nz; i++) k[c->I[i]] += c->V[i];
}

/* ------------------------------------------------------------------------- */
/* Serial kernels: serial/SerialCG.cpp.                                      */

void orc_matvec_coo(int N, int nz, const int *I, const int *J, const double *V,
                    const double *x, double *y) {
  memset(y, 0, sizeof(double) * (size_t)N);
  for (int i = 0; i < nz; i++) y[I[i]] += V[i] * x[J[i]];
}

void orc_matvec_crs(int N, const int *ptr, const int *index,
                    const double *value, const double *x, double *y) {
  for (int i = 0; i < N; i++) {
    double tmp = 0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) tmp += value[j] * x[index[j]];
    y[i] = tmp;
  }
}

void orc_matvec_ell(int N, const int *length, const int *index,
                    const double *data, const double *x, double *y) {
  for (int i = 0; i < N; i++) {
    double tmp = 0;
    for (int j = 0; j < length[i]; j++) {
      size_t k = (size_t)j * (size_t)N + (size_t)i;
      tmp += data[k] * x[index[k]];
    }
    y[i] = tmp;
  }
}

void orc_axpy(int N, double a, const double *x, double *y) {
  for (int i = 0; i < N; i++) y[i] += a * x[i];
}

void orc_xpay(int N, const double *x, double a, double *y) {
  for (int i = 0; i < N; i++) y[i] = x[i] + a * y[i];
}

double orc_dot(int N, const double *a, const double *b) {
  double res = 0;
  for (int i = 0; i < N; i++) res += a[i] * b[i];
  return res;
}

void orc_jacobi_apply(int N, const double *C, const double *x, double *y) {
  for (int i = 0; i < N; i++) y[i] = C[i] * x[i];
}

static void matvec(const orc_matrix *A, const double *x, double *y) {
  switch (A->format) {
  case ORC_FMT_COO:
    orc_matvec_coo(A->N, A->nz, A->I, A->J, A->V, x, y);
    break;
  case ORC_FMT_CRS:
    orc_matvec_crs(A->N, A->ptr, A->index, A->value, x, y);
    break;
  default:
    orc_matvec_ell(A->N, A->length, A->index, A->data, x, y);
    break;
  }
}

/* ------------------------------------------------------------------------- */
/* CG::solve (CG.cpp:284-385).                                               */

int orc_cg_solve(const orc_matrix *A, const double *C, const double *k,
                 double *x, int maxIterations, double tolerance,
                 double *residualOut) {
  int N = A->N;
  size_t bytes = sizeof(double) * (size_t)(N > 0 ? N : 1);
  double *p = (double *)malloc(bytes), *q = (double *)malloc(bytes);
  double *r = (double *)malloc(bytes), *z = (double *)malloc(bytes);
  double rho, rho_old, r2, nrm2_0, dot_pq, a, b;
  double residual = 0;
  int iteration;

  /* r(0) = k - A x(0) */
  matvec(A, x, r);
  orc_xpay(N, k, -1.0, r);
  if (!C)
    memcpy(p, r, sizeof(double) * (size_t)N);
  else
    orc_jacobi_apply(N, C, r, p);
  r2 = orc_dot(N, r, r);
  nrm2_0 = sqrt(r2);
  rho = C ? orc_dot(N, p, r) : r2;

  for (iteration = 0; iteration < maxIterations; iteration++) {
    matvec(A, p, q);
    dot_pq = orc_dot(N, p, q);
    a = rho / dot_pq;
    orc_axpy(N, a, p, x);
    orc_axpy(N, -a, q, r);
    r2 = orc_dot(N, r, r);
    residual = sqrt(r2) / nrm2_0;
    if (residual <= tolerance) {
      iteration++;
      break;
    }
    rho_old = rho;
    if (!C) {
      rho = r2;
    } else {
      orc_jacobi_apply(N, C, r, z);
      rho = orc_dot(N, r, z);
    }
    b = rho / rho_old;
    orc_xpay(N, C ? z : r, b, p);
  }

  free(p);
  free(q);
  free(r);
  free(z);
  if (residualOut) *residualOut = residual;
  return iteration;
}

/* CG::check (CG.cpp:387-408). */
int orc_check_ones(int N, const double *x, double checkTolerance) {
  int errors = 0;
  for (int i = 0; i < N; i++)
    if (fabs(x[i] - 1.0) > checkTolerance) errors++;
  return errors;
}

/* ------------------------------------------------------------------------- */
/* Mixed-precision iterative refinement (no reference counterpart).          */

static double dot_f32_acc64(int N, const float *a, const float *b) {
  double s = 0;
  for (int i = 0; i < N; i++) s += (double)a[i] * (double)b[i];
  return s;
}

int orc_mixed_ir_solve(int N, const int *ptr, const int *index,
                       const double *value, const double *C, const double *b,
                       double *x, int maxIterations, double tolerance,
                       double innerTol, int maxOuter, int *outerOut,
                       double *trueResidual) {
  int nnz = ptr[N];
  float *vf = (float *)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
  float *Cf = (float *)malloc(sizeof(float) * (size_t)(N > 0 ? N : 1));
  for (int j = 0; j < nnz; j++) vf[j] = (float)value[j];
  for (int i = 0; i < N; i++) Cf[i] = (float)C[i];
  size_t fb = sizeof(float) * (size_t)(N > 0 ? N : 1);
  float *d = (float *)malloc(fb), *r = (float *)malloc(fb);
  float *p = (float *)malloc(fb), *q = (float *)malloc(fb);
  double *r64 = (double *)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));

  double nb = sqrt(orc_dot(N, b, b));
  int total = 0, outer = 0;
  double rel = 0;
  for (;;) {
    /* FP64 true residual r = b - A x. */
    orc_matvec_crs(N, ptr, index, value, x, r64);
    for (int i = 0; i < N; i++) r64[i] = b[i] - r64[i];
    double nr = sqrt(orc_dot(N, r64, r64));
    rel = nb > 0 ? nr / nb : 0;
    if (rel <= tolerance || outer >= maxOuter || total >= maxIterations) break;
    outer++;

    /* Inner FP32 Jacobi-PCG on A d = r / ||r||. */
    double tolIn = 0.5 * tolerance / rel;
    if (tolIn < innerTol) tolIn = innerTol;
    double inv = 1.0 / nr;
    for (int i = 0; i < N; i++) {
      r[i] = (float)(r64[i] * inv);
      d[i] = 0.0f;
      p[i] = Cf[i] * r[i];
    }
    double rho = dot_f32_acc64(N, r, p);
    double nrm0 = sqrt(dot_f32_acc64(N, r, r));
    while (total < maxIterations) {
      for (int i = 0; i < N; i++) {
        float t = 0.0f;
        for (int j = ptr[i]; j < ptr[i + 1]; j++) t += vf[j] * p[index[j]];
        q[i] = t;
      }
      double pq = dot_f32_acc64(N, p, q);
      float a = (float)(rho / pq);
      for (int i = 0; i < N; i++) {
        d[i] += a * p[i];
        r[i] -= a * q[i];
      }
      total++;
      double rr = dot_f32_acc64(N, r, r);
      if (sqrt(rr) / nrm0 <= tolIn) break;
      double rz = 0;
      for (int i = 0; i < N; i++) rz += (double)r[i] * (double)(Cf[i] * r[i]);
      float beta = (float)(rz / rho);
      rho = rz;
      for (int i = 0; i < N; i++) p[i] = Cf[i] * r[i] + beta * p[i];
    }
    for (int i = 0; i < N; i++) x[i] += nr * (double)d[i];
  }

  free(vf);
  free(Cf);
  free(d);
  free(r);
  free(p);
  free(q);
  free(r64);
  if (outerOut) *outerOut = outer;
  if (trueResidual) *trueResidual = rel;
  return total;
}
