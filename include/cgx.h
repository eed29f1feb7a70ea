/*
 * cgx.h -- C ABI of libcgb200, the B200 (sm_100a) conjugate-gradient engine.
 *
 * The reference (hahnjo/CGxx) plugs a programming model into its solver by
 * deriving from the abstract class CG (CG.h:19-293) and overriding its
 * per-kernel virtual methods (CG.h:180-237); the CUDA plug-in is
 * cuda/CGCUDA.cu. Every entry point below names the reference method it
 * replaces. A plug-in that binds this library needs nothing but these plain C
 * declarations: no CUDA, torch or C++ types cross the boundary.
 *
 * Conventions
 *   - Every function returns a cgx_status; CGX_SUCCESS is 0. On failure
 *     cgx_last_error() returns a message for the calling thread. (The
 *     reference instead prints "CUDA error: ..." and calls exit(1),
 *     cuda/utils.h:10-15; the host CG class of this project converts a
 *     failed status into exactly that behaviour.)
 *   - Host pointers are ordinary (pageable or pinned) host memory; the
 *     library copies from/to them. Pinned buffers make the copies faster.
 *   - A handle is bound to one device and one CUDA stream and must be used by
 *     one host thread at a time, like the reference's single-threaded CG.
 *   - Matrices use 0-based int32 indices and double values, laid out exactly
 *     as the reference's MatrixCRS / MatrixELL / MatrixCOO (Matrix.h:22-103).
 */
#ifndef CGX_H
#define CGX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGX_VERSION_MAJOR 1
#define CGX_VERSION_MINOR 0

typedef struct cgx_handle cgx_handle;

typedef enum cgx_status {
  CGX_SUCCESS = 0,
  CGX_ERROR_INVALID_ARGUMENT = 1, /* bad pointer, size, enum or matrix data */
  CGX_ERROR_INVALID_STATE = 2,    /* e.g. solve before a matrix is uploaded */
  CGX_ERROR_UNSUPPORTED = 3,      /* format/preconditioner/precision combo */
  CGX_ERROR_CUDA = 4,             /* a CUDA runtime call failed */
  CGX_ERROR_OUT_OF_MEMORY = 5,    /* device allocation failed */
  CGX_ERROR_DEVICE = 6,           /* a device-side check failed (see text) */
  CGX_ERROR_IO = 7,               /* MatrixMarket file could not be read */
  CGX_ERROR_NUMERICAL = 8         /* NaN/Inf or breakdown that ended a solve */
} cgx_status;

/* CG::Vector (CG.h:22-35), same order and meaning. */
typedef enum cgx_vector {
  CGX_VECTOR_K = 0, /* right-hand side */
  CGX_VECTOR_X = 1, /* solution */
  CGX_VECTOR_P = 2, /* search direction */
  CGX_VECTOR_Q = 3, /* A p */
  CGX_VECTOR_R = 4, /* residual */
  CGX_VECTOR_Z = 5  /* preconditioned residual */
} cgx_vector;

/* CG::MatrixFormat (CG.h:38-47). */
typedef enum cgx_format {
  CGX_FORMAT_COO = 0,
  CGX_FORMAT_CRS = 1,
  CGX_FORMAT_ELL = 2
} cgx_format;

/* CG::Preconditioner (CG.h:50-55), plus the learned factor G G^T + eps I. */
typedef enum cgx_preconditioner {
  CGX_PRECONDITIONER_NONE = 0,
  CGX_PRECONDITIONER_JACOBI = 1,
  CGX_PRECONDITIONER_LEARNED = 2
} cgx_preconditioner;

typedef enum cgx_precision {
  CGX_PRECISION_FP64 = 0, /* the reference's arithmetic (def.h:6) */
  CGX_PRECISION_MIXED = 1 /* FP32 inner PCG inside FP64 refinement */
} cgx_precision;

typedef enum cgx_loop {
  CGX_LOOP_GRAPH = 0,   /* whole solve = one CUDA graph with a while node;
                           the mixed paths on the band form run their inner
                           solves as persistent launches below (PERSISTENT up
                           to 1.3M rows, PERSISTENT_SPLIT beyond), which
                           measured faster at every size */
  CGX_LOOP_CHUNKED = 1, /* graph of a fixed number of iterations, host polls */
  CGX_LOOP_KERNELS = 2, /* one launch per fused kernel, each timed by events */
  CGX_LOOP_PERSISTENT = 3, /* mixed paths on the band form (the 7- and
                           5-point stencils, any size): each inner solve is
                           one cooperative launch whose fused phases (three
                           per learned iteration, two per Jacobi one) meet at
                           grid-wide barriers; other solves run as GRAPH */
  CGX_LOOP_PERSISTENT_SPLIT = 4 /* the same launch with one phase per kernel
                           of the GRAPH iteration (five learned, three
                           Jacobi) and no value formed twice; also on SELL-U
                           inner products whose slices are all uniform (the
                           27-point stencils), where GRAPH takes it too */
} cgx_loop;

/* Solver settings: the reference's CG_* environment switches
 * (CG.cpp:35-149) plus this library's own. */
typedef struct cgx_options {
  int max_iterations;      /* CG_MAX_ITER, > 0 (CG.h:67, default 1000) */
  double tolerance;        /* CG_TOLERANCE, > 0 (CG.h:70, default 1e-9) */
  int preconditioner;      /* cgx_preconditioner (default JACOBI) */
  int precision;           /* cgx_precision (default FP64) */
  int loop;                /* cgx_loop (default GRAPH) */
  double inner_tolerance;  /* MIXED: floor of the inner relative tolerance (3e-6) */
  int max_outer;           /* MIXED: limit on refinement steps */
  int compute_true_residual; /* FP64 ||k - A x|| / ||k|| after the solve */
} cgx_options;

typedef struct cgx_result {
  int iterations;        /* as printed by CG::printSummary (CG.cpp:424);
                            MIXED: total inner iterations */
  double residual;       /* FP64: recurrence residual ||r|| / ||r0||
                            (CG.cpp:350); MIXED: FP64 true residual */
  double true_residual;  /* ||k - A x|| / ||k|| in FP64 if requested, else -1 */
  int converged;         /* residual <= tolerance */
  int outer_iterations;  /* MIXED: refinement steps; 0 otherwise */
  double solve_ms;       /* device time of the solve (CUDA events) */
  /* CGX_LOOP_KERNELS only: device time per fused kernel class (ms) and the
   * number of launches of each; zero in the other loop modes:
   * (q = A p | r update, and for the learned path the apply z = G G^T r +
   * eps C r | p update). */
  double spmv_ms, update_ms, direction_ms;
  int spmv_launches, update_launches, direction_launches;
  int fell_back;         /* MIXED: an FP32 refinement step broke down or
                            stalled (its FP64 true residual was NaN/Inf or
                            fell by less than half); it was undone and the
                            solve finished with plain FP64 Jacobi-CG from the
                            restored x, with a budget of max_iterations of its
                            own. iterations then counts both parts. A system
                            that no budget solves (e.g. singular and
                            inconsistent) ends with status CGX_SUCCESS and
                            converged = 0. */
  int inner_form;        /* MIXED: how the inner solves ran: 0 per-iteration
                            kernels, 1 fused persistent launches, 2 split
                            persistent launches on the band form, 3 split
                            persistent launches on SELL-U (cgx_loop) */
  int inner_launches;    /* MIXED, inner_form 1 or 2: persistent launches */
  double inner_ms;       /* MIXED, inner_form 1 or 2: their device time (CUDA
                            events around each launch) */
} cgx_result;

/* Library ------------------------------------------------------------------ */

void cgx_version(int *major, int *minor);
const char *cgx_status_string(cgx_status s);
/* Message of the last failed call on this thread ("" if none). */
const char *cgx_last_error(void);
/* Number of CUDA devices visible (0 on a machine without a GPU). */
cgx_status cgx_device_count(int *count);
cgx_status cgx_default_options(cgx_options *opts);

/* Handle: replaces the device bookkeeping of CGCUDABase::Device
 * (cuda/CGCUDABase.h:17-90) and checkedSetDevice(0) in CGCUDA::init
 * (cuda/CGCUDA.cu:29-36). `device` is a CUDA ordinal. */
cgx_status cgx_create(cgx_handle **out, int device);
cgx_status cgx_destroy(cgx_handle *h);
/* Uses an existing cudaStream_t (passed as void*) for all work; NULL
 * restores the handle's own stream. */
cgx_status cgx_set_stream(cgx_handle *h, void *stream);
cgx_status cgx_synchronize(cgx_handle *h);

/* Data transfer: CGCUDA::doTransferTo (cuda/CGCUDA.cu:38-75) and
 * CGCUDABase::allocateAndCopyMatrixDataCRS/ELL (cuda/CGCUDABase.cu:5-37).
 * Uploading a matrix (re)allocates every device vector for its N; K, X are
 * zeroed. Arrays are validated (ptr monotone from 0 to nz, indices in
 * [0, N)); invalid data returns CGX_ERROR_INVALID_ARGUMENT. */
cgx_status cgx_upload_crs(cgx_handle *h, int N, int nz, const int *ptr,
                          const int *index, const double *value);
/* ELL as in MatrixDataELL (Matrix.h:74-87): column-major, element (i, j) at
 * j*N + i, length[i] entries used per row (0 <= length[i] <= maxNz, summing
 * to nz), maxNz slots per row. The paths
 * that read rows (mixed, learned, cgx_jacobi_from_matrix) build a CRS copy
 * of it on the device on first use. */
cgx_status cgx_upload_ell(cgx_handle *h, int N, int nz, int maxNz,
                          const int *length, const int *index,
                          const double *data);
/* COO as in MatrixCOO (Matrix.h:22-31), entries in file order. The device
 * groups it by row (cgx_upload_coo_as), each row's entries in file order
 * (the order in which serial/SerialCG.cpp:79-85 adds them), in the CRS
 * layout. */
cgx_status cgx_upload_coo(cgx_handle *h, int N, int nz, const int *I,
                          const int *J, const double *V);
/* MatrixCOO (Matrix.h:22-31, entries in file order) converted on the device
 * into `format` (a cgx_format): the reference's DataMatrix<CRS>::convert
 * (Matrix.cpp:203-228) and DataMatrix<ELL>::convert (Matrix.cpp:339-361),
 * which run on its host, and the row grouping of its COO product
 * (serial/SerialCG.cpp:79-85). A stable radix sort by row on the device
 * keeps every row's entries in file order, so the CRS and ELL arrays are the
 * reference's bit for bit. Row or column indices outside [0, N) return
 * CGX_ERROR_INVALID_ARGUMENT. cgx_upload_coo is this call with
 * CGX_FORMAT_COO. */
cgx_status cgx_upload_coo_as(cgx_handle *h, int N, int nz, const int *I,
                             const int *J, const double *V, int format);
/* Read-back of the device's matrix (no counterpart in the reference; for
 * tests and tools): the row layout (ptr: N + 1, index and value: nz; built
 * on the device from an ELL upload if needed), and, for ELL uploads, the
 * reference's column-major arrays (index and data: max_nz * N, element
 * (i, j) at j * N + i, padding slots 0). Each pointer may be NULL. */
cgx_status cgx_download_crs(cgx_handle *h, int *ptr, int *index, double *value);
cgx_status cgx_download_ell(cgx_handle *h, int *max_nz, int *length,
                            int *index, double *data);
/* Jacobi::C (Preconditioner.h:12-25), N doubles. */
cgx_status cgx_upload_jacobi(cgx_handle *h, const double *C);
/* Computes C[i] = 1 / A_ii on the device from the uploaded matrix, with the
 * semantics of Jacobi::init (Preconditioner.cpp:13-23): the last diagonal
 * entry of a row in file order wins; a row without one gets C = 0. */
cgx_status cgx_jacobi_from_matrix(cgx_handle *h);
cgx_status cgx_set_vector(cgx_handle *h, cgx_vector v, const double *host);
/* CGCUDA::doTransferFrom (cuda/CGCUDA.cu:77-112) for one vector. */
cgx_status cgx_get_vector(cgx_handle *h, cgx_vector v, double *host);
cgx_status cgx_fill_vector(cgx_handle *h, cgx_vector v, double value);
cgx_status cgx_matrix_info(cgx_handle *h, int *N, int *nz, int *format);

/* Per-kernel interface, one entry per pure virtual of CG (CG.h:224-237),
 * operating on the device-resident vectors. */
cgx_status cgx_copy(cgx_handle *h, cgx_vector dst, cgx_vector src); /* cpy */
cgx_status cgx_matvec(cgx_handle *h, cgx_vector x, cgx_vector y);   /* y = A x */
cgx_status cgx_axpy(cgx_handle *h, double a, cgx_vector x,
                    cgx_vector y);                                 /* y += a x */
cgx_status cgx_xpay(cgx_handle *h, cgx_vector x, double a,
                    cgx_vector y);                          /* y = x + a y */
cgx_status cgx_dot(cgx_handle *h, cgx_vector a, cgx_vector b,
                   double *result);                         /* <a, b> */
cgx_status cgx_apply_jacobi(cgx_handle *h, cgx_vector x,
                            cgx_vector y); /* y = C o x */

/* CG::solve (CG.cpp:284-385) as one device-resident solve: r = k - A x,
 * then PCG until ||r|| / ||r0|| <= tolerance or max_iterations, with every
 * scalar kept on the device. Starts from the current X (the reference's
 * resetX sets it to 0, CG.cpp:272-275) and leaves the solution in X. */
cgx_status cgx_solve(cgx_handle *h, const cgx_options *opts,
                     cgx_result *result);

/* Learned preconditioner M^-1 = G G^T + eps D^-1 (no counterpart in the
 * reference; it extends CG_PRECONDITIONER beyond none/jacobi). G is lower
 * triangular on the pattern of tril(A); its values come from a small
 * message-passing network (3 layers, width 32, BF16 tensor cores with FP32
 * accumulation) that reads the Jacobi-scaled matrix. The arithmetic is stated
 * in oracle/gnn_oracle.py. Used by cgx_solve with
 * preconditioner = CGX_PRECONDITIONER_LEARNED and precision = MIXED. */
typedef struct cgx_gnn cgx_gnn;
int cgx_gnn_param_count(void);
/* params: cgx_gnn_param_count() floats in the oracle's layout, or NULL (0). */
cgx_status cgx_gnn_create(cgx_gnn **out, int device, const float *params);
cgx_status cgx_gnn_destroy(cgx_gnn *g);
cgx_status cgx_gnn_set_params(cgx_gnn *g, const float *params);
cgx_status cgx_gnn_get_params(cgx_gnn *g, float *params);
/* Replaces the values of the uploaded CRS matrix (same pattern); `value`
 * may be host or device memory. */
cgx_status cgx_update_crs_values(cgx_handle *h, const double *value);
/* Builds the Jacobi-scaled graph of the uploaded matrix (needs positive
 * diagonal entries and a structurally symmetric pattern). After
 * cgx_update_crs_values it only recomputes the scaled values. */
cgx_status cgx_learned_setup(cgx_handle *h);
/* Network inference: G and G^T for the current matrix, eps >= 0. */
cgx_status cgx_learned_factor(cgx_handle *h, cgx_gnn *g, double eps);
/* Unscaled factor Ghat = D^1/2 G on its pattern (arrays of *nnzL entries,
 * each optional). */
cgx_status cgx_learned_get_factor(cgx_handle *h, int *nnzL, float *ghat,
                                  int *rows, int *cols);
/* z = G (G^T r) + eps C r, the learned preconditioner as the inner solve
 * applies it (BF16 factor values, FP32 vectors), on N host floats (no
 * counterpart in the reference; it exposes that product to tests). Needs
 * cgx_learned_factor and the Jacobi vector C; overwrites the inner vectors
 * and the solver scalars. */
cgx_status cgx_learned_apply(cgx_handle *h, const float *r, float *z);
/* Probe recipe of the network's training (no counterpart in the reference),
 * for the 8 probe columns: the last `residual_cols` are the handle's
 * residual snapshots (cgx_learned_capture_residual; they must exist for the
 * current values); the `smooth_cols` before them are Rademacher columns
 * that take `smooth_steps` damped-Jacobi steps V <- V - (2/3) Ahat V on the
 * Jacobi-scaled matrix and are multiplied by `smooth_scale`; the rest are
 * Rademacher columns from the seed. Both kinds weight the loss toward the
 * smooth end of the spectrum that limits CG. Default 0, 0, 1, 0 (plain
 * Rademacher probes). */
cgx_status cgx_gnn_set_probes(cgx_gnn *g, int smooth_steps, int smooth_cols,
                              float smooth_scale, int residual_cols);
/* Residual snapshot for the probe recipe (no counterpart in the reference):
 * r = k - A x of the current K and X in FP64 (x typically an iterate of a
 * solve the caller ran), Jacobi-scaled (D^-1/2 r) and normalized to unit
 * RMS, stored as probe column `col` (0..7) of the handle's learned state.
 * Snapshots are dropped when cgx_learned_setup takes new values. */
cgx_status cgx_learned_capture_residual(cgx_handle *h, int col);
/* Hutchinson loss ||(Ghat^T Ahat Ghat - I) V||_F^2 / (N S) for S = 8 probe
 * columns (probes: N*8 floats, node-major, or NULL for the network's probe
 * recipe from `seed`) and its gradient w.r.t. the parameters (grad may be
 * NULL). */
cgx_status cgx_gnn_loss_grad(cgx_gnn *g, cgx_handle *h, const float *probes,
                             unsigned long long seed, float *loss,
                             float *grad);
/* One Adam step on the network's probe recipe from `seed`; *loss
 * (optional) is the loss before the step. */
cgx_status cgx_gnn_train_step(cgx_gnn *g, cgx_handle *h,
                              unsigned long long seed, float lr, float *loss);

/* FP64 ||k - A x|| / ||k|| of the current X. */
cgx_status cgx_true_residual(cgx_handle *h, double *rel);

/* Device time of the solver's SpMV alone (no counterpart in the
 * reference): `reps` back-to-back launches of the fused product the solve
 * runs (FP64: q = A p with <p,q> on the uploaded format; MIXED: the FP32
 * inner q = A p with <p,q> on the inner form) are captured into a CUDA
 * graph and timed with CUDA events
 * on the handle's stream after one untimed launch of the graph;
 * *us_per_launch is the average. Uses the current P (FP64) or inner vectors
 * (MIXED) and overwrites Q, the inner vectors and the solver scalars of the
 * last solve. */
cgx_status cgx_time_spmv(cgx_handle *h, cgx_precision precision, int reps,
                         double *us_per_launch);

/* Diagnostics of failure detection (no counterpart in the reference): runs
 * a kernel whose wait can never complete, with a short limit (a few
 * milliseconds): which = 0, the grid barrier of the persistent inner solves;
 * which = 1, the mbarrier wait of the bulk-copy staged products. The wait
 * gives up, the kernel sets its error bit (*error_bits receives the
 * solver state's error bits: 4 grid barrier, 1 bulk-copy wait) and returns,
 * and the call returns CGX_ERROR_DEVICE as a solve would; the handle stays
 * usable. Needs a matrix (for the solver scratch). */
cgx_status cgx_check_wait_timeout(cgx_handle *h, int which, int *error_bits);

/* Symmetric band form of A's FP32 copy (no counterpart in the reference):
 * when A is symmetric and all its column offsets col - row form one
 * symmetric set with at most 4 non-negative members (the 7-point
 * structured-grid stencil: 0, 1, n, n^2), the inner SpMV stores per row
 * only the values at those offsets (the diagonal and the upper half) and
 * reads each lower entry from the row above that holds it.
 * *stored_offsets = that count, or 0 when the inner SpMV uses another form
 * (or the FP32 copy is not built yet); offsets (NULL, or room for 4)
 * receives them, ascending from 0. */
cgx_status cgx_inner_band(cgx_handle *h, int *stored_offsets, int *offsets);

/* y = A x by the inner FP32 SpMV of the mixed and learned paths, on
 * whichever form it uses (no counterpart in the reference; it exposes that
 * product to tests): x and y are N host floats. Builds the FP32 copy if
 * needed; overwrites the inner p and q and the solver scalars. */
cgx_status cgx_inner_matvec(cgx_handle *h, const float *x, float *y);

/* Layout of A's FP32 copy used by the inner SpMV of the mixed and learned
 * paths (built by the first mixed solve; no counterpart in the reference):
 * rows in slices of 32, *slices in all, *uniform_slices of them storing one
 * column offset per slot for all 32 rows (no per-entry index), *value_slots
 * FP32 values including zero padding. *value_slots = 0: the inner SpMV uses
 * FP32 CRS (not built yet, or the layout's indices would not fit in int). */
cgx_status cgx_inner_layout(cgx_handle *h, long long *value_slots,
                            long long *uniform_slices, long long *slices);

/* MatrixMarket I/O (MatrixCOO::MatrixCOO, Matrix.cpp:13-111). Reads a
 * `matrix coordinate real general|symmetric` file into newly malloc'ed
 * arrays (free them with cgx_free) with the reference's entry order:
 * symmetric off-diagonal entries are mirrored into the next slot. The file
 * is parsed by several host threads. Returns CGX_ERROR_IO with the
 * reference's message on the conditions where it calls exit(1). */
cgx_status cgx_mtx_read(const char *path, int *N, int *nz, int **I, int **J,
                        double **V);
/* Writes the lower triangle (row >= col) of a CRS matrix as a symmetric
 * MatrixMarket file with 17 significant digits (round-trips exactly). */
cgx_status cgx_mtx_write_symmetric_crs(const char *path, int N,
                                       const int *ptr, const int *index,
                                       const double *value);
void cgx_free(void *p);

/* Dot product <a, b> of two device vectors of n doubles, written to *result
 * (device memory), for callers that cannot allocate device memory: code
 * running under a framework that owns all device memory, or a loop whose
 * rules forbid allocation after start-up. It needs no handle and calls no
 * allocating routine; its scratch (one partial sum per 4096-element chunk)
 * lives in a fixed 512 KiB array in the library image, held by every GPU that
 * loads the library until exit. Hence n <= 268,435,456; larger n returns
 * CGX_ERROR_INVALID_ARGUMENT.
 *   - Works on the calling thread's current device, on `stream` (a
 *     cudaStream_t; NULL = the legacy default stream); asynchronous.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 *   - All calls share the one array: calls that overlap on the GPU (different
 *     streams, or several host threads) race and give wrong results.
 *   - The looked-up address is kept for the life of the process. After
 *     cudaDeviceReset on a device, the library image may load at another
 *     address, so calls on that device are then invalid.
 * Deterministic: the result depends only on a, b and n.
 * Has no counterpart in the reference. */
cgx_status cgx_dot_noalloc(const double *a, const double *b, int n,
                           double *result, void *stream);

/* Page-locked host memory for vectors that cross the boundary every solve
 * (the reference pins x: CGCUDABase::allocateX, cuda/CGCUDABase.h:101-104).
 * Free with cgx_host_free. */
cgx_status cgx_host_alloc(void **p, size_t bytes);
cgx_status cgx_host_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* CGX_H */
