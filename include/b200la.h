/*
 * b200la -- B200-native (sm_100a) local linear algebra for HiFlow3's
 * Jacobi-preconditioned CG hot path.  C ABI: opaque handles, plain pointers
 * and sizes, int status codes (0 = ok, < 0 = error, never exit()).
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the HiFlow3 source tree, src/).  A reference binding
 * registers these behind lmp's lVector / lMatrix / lPreconditioner and the
 * linear_solver CG interface.
 *
 * Threading: a context is used by one host thread at a time (the reference's
 * lmp objects are not thread-safe either, common/timer.h:28).  All device
 * work of a context is ordered on its stream.  Calls that return a host
 * value (dot, norm, download, solve results) synchronise that stream, as the
 * reference's blocking cuBLAS calls do (lmp/cuda/GPUblas_lvector.cu:196-211).
 */
#ifndef B200LA_H
#define B200LA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b200la_ctx_s *b200la_ctx;
typedef struct b200la_vec_s *b200la_vec;
typedef struct b200la_mat_s *b200la_mat;
typedef struct b200la_cg_s *b200la_cg;
typedef struct b200la_mp_s *b200la_mp;
typedef struct b200la_batch_s *b200la_batch;

/* ---- status codes --------------------------------------------------------
 * The reference reports errors by LOG_ERROR + exit(-1)/quit_program()
 * (lmp/cuda/cuda_utils.h:24-55, lmp/cuda/GPUscalar_csr_lmatrix.cu:73-80);
 * here every failure is a negative return and a message in
 * b200la_last_error(). */
#define B200LA_OK 0
#define B200LA_ERR_INVALID (-1)     /* bad argument: null handle, size mismatch */
#define B200LA_ERR_CUDA (-2)        /* CUDA runtime error */
#define B200LA_ERR_NOMEM (-3)       /* device allocation failed */
#define B200LA_ERR_DTYPE (-4)       /* dtype mismatch between operands */
#define B200LA_ERR_MATRIX (-5)      /* malformed CSR, or missing diagonal */
#define B200LA_ERR_TIMEOUT (-6)     /* a bounded device-side wait expired */
#define B200LA_ERR_UNSUPPORTED (-7) /* valid request this build does not do */

/* value types: la_global.h templates on double / float */
#define B200LA_F64 0
#define B200LA_F32 1

/* iterate states: IterateControl::State (common/iterate_control.h) */
#define B200LA_ITERATE 0
#define B200LA_SUCCESS_ABS 1
#define B200LA_SUCCESS_REL 2
#define B200LA_FAIL_DIV 3
#define B200LA_FAIL_MAXITS 4
#define B200LA_FAIL_BREAKDOWN 5 /* p.Ap == 0 or not finite (no reference analogue) */

/* linear solver states: LinearSolverState (linear_solver/preconditioner.h:33) */
#define B200LA_SOLVER_SUCCESS 0
#define B200LA_SOLVER_EXCEEDED 1
#define B200LA_SOLVER_ERROR 2

/* SpMV storage formats (la_global.h:56 MATRIX_FORMAT has DENSE, CSR, COO, ELL) */
#define B200LA_FMT_CSR 1  /* CSR, a group of `lanes` threads per row */
#define B200LA_FMT_SELL 4 /* SELL-C-sigma (C = 32 and sigma = 1 unless b200la_mat_to_sell says otherwise) */
#define B200LA_FMT_SELL16 5 /* SELL-32 with columns stored as int16 offsets from the row
                             (banded matrices: every |col - row| <= 32767) */
#define B200LA_FMT_STENCIL 6 /* values-only sliced ELL: square matrices whose rows' columns all
                              lie in one list of 9 or 27 offsets from the row (structured-grid
                              Q1 matrices); no column storage */

/* ---- library / context ---------------------------------------------------
 * replaces init_platform_gpu (lmp/cuda/platform_management_gpu.cu:78-143) */
const char *b200la_version(void);
const char *b200la_last_error(void); /* message of this thread's last error */
int b200la_ctx_create(int device, b200la_ctx *out);
int b200la_ctx_destroy(b200la_ctx ctx);
/* Use an external cudaStream_t (NULL: the context's own stream). */
int b200la_ctx_set_stream(b200la_ctx ctx, void *stream);
int b200la_ctx_get_stream(b200la_ctx ctx, void **stream);
/* Device loops (the solvers' iterations, the batch's passes) run as CUDA-graph
 * WHILE nodes; with on = 0 the same kernels launch one by one from a host
 * loop on this context (the environment variable B200LA_GRAPHS=0 sets the
 * default of new contexts).  Results are the same bits either way; a host
 * loop lets a profiler or a launch record see every kernel.  Takes effect at
 * the next solve or run. */
int b200la_ctx_set_graphs(b200la_ctx ctx, int on);
int b200la_ctx_synchronize(b200la_ctx ctx);
int b200la_ctx_num_sms(b200la_ctx ctx, int *out);

/* ---- vectors: lVector<T> (lmp/lvector.h:38-321), GPU_lVector
 * (lmp/cuda/lvector_gpu.cc) ---------------------------------------------- */
/* Init(size, name): device buffer of n values, zero-filled (lvector_gpu.cc:90-104) */
int b200la_vec_create(b200la_ctx ctx, int64_t n, int dtype, b200la_vec *out);
/* Non-owning view of an existing device buffer (GPU_lVector::buffer, lvector_gpu.h:118). */
int b200la_vec_wrap(b200la_ctx ctx, int64_t n, int dtype, void *device_ptr, b200la_vec *out);
int b200la_vec_destroy(b200la_vec v);                              /* Clear + delete */
int b200la_vec_info(b200la_vec v, int64_t *n, int *dtype, void **device_ptr);
/* SetBlockValues(0, n, host) / GetBlockValues(0, n, host) (lvector.h:113-124) */
int b200la_vec_upload(b200la_vec v, const void *host, int64_t n);
int b200la_vec_download(b200la_vec v, void *host, int64_t n);
/* SetValues / GetValues at host index lists (lvector.h:91-103) */
int b200la_vec_set_values(b200la_vec v, const int *index, const void *values, int size);
int b200la_vec_get_values(b200la_vec v, const int *index, void *values, int size);
int b200la_vec_zeros(b200la_vec v);                                /* Zeros */
int b200la_vec_copy(b200la_vec dst, b200la_vec src);               /* CopyFrom */
int b200la_vec_cast(b200la_vec dst, b200la_vec src);               /* CastFrom */
int b200la_vec_dot(b200la_vec a, b200la_vec b, double *out);       /* Dot */
int b200la_vec_norm2(b200la_vec v, double *out);                   /* Norm2 */
int b200la_vec_axpy(b200la_vec y, b200la_vec x, double alpha);     /* y.Axpy(x, a): y += a x */
int b200la_vec_scaleadd(b200la_vec y, double alpha, b200la_vec x); /* y.ScaleAdd(a, x): y = a y + x */
int b200la_vec_scale(b200la_vec v, double alpha);                  /* Scale */
int b200la_vec_elementwise_mult(b200la_vec y, b200la_vec x);       /* ElementWiseMult: y .*= x */
/* partial_replace_subvector / partial_add_subvector (lvector.h:175-190):
 * dst[dst_start + i] = src[src_start + i] (add = 0) or += weight * src[...]
 * (add = 1) for i < n; the ranges may start anywhere. */
int b200la_vec_range_update(b200la_vec dst, int64_t dst_start, b200la_vec src, int64_t src_start, int64_t n,
                            int add, double weight);
/* Device halo of a row-partitioned vector (CoupledVector::SendBorder /
 * ReceiveGhost, linear_algebra/coupled_vector.cc:890-973, which stage the
 * values through host buffers and MPI): gather out[k] = src[idx[k]] into a
 * device send buffer, scatter dst[idx[k]] = in[k] from a device receive
 * buffer; idx is a device int32 array of n indices (in range: not checked on
 * the device), out/in device buffers of n values of the vector's dtype.
 * Stream-ordered on the context stream, so a collective on the same stream
 * (or one that waits on it) moves the buffers in between. */
int b200la_vec_gather(b200la_vec src, const int *idx, int64_t n, void *out);
int b200la_vec_scatter(b200la_vec dst, const int *idx, int64_t n, const void *in);

/* Dot product that allocates nothing (no counterpart in the reference; its
 * lmp Dot is the entry above).  For callers that cannot call cudaMalloc:
 * cudaMalloc/cudaFree can stall the whole device while overlapped work is in
 * flight, and applications that give all device memory to their own pool, or
 * run this library as a plug-in under a fixed quota, may not allocate
 * outside it.  x and y are device buffers of n values of dtype on the current
 * device; the total is written to *out (host) after `stream` (a
 * cudaStream_t, NULL = legacy default stream) is synchronised.  The reduction
 * scratch is one fixed ~32 KB __device__ array that every GPU loading the
 * library keeps until exit, so n is limited to 16,777,216 elements; larger n
 * is rejected with B200LA_ERR_UNSUPPORTED.  The first call on a device (and
 * the first after cudaDeviceReset replaced its context) looks up the array's
 * device address and caches it; make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller. */
int b200la_dot_noalloc(const void *x, const void *y, int64_t n, int dtype, void *stream,
                       double *out);

/* ---- matrices: lMatrix<T> / CSR_lMatrix<T> (lmp/lmatrix.h:39-468),
 * GPU_CSR_lMatrix (lmp/cuda/lmatrix_csr_gpu.cc) ----------------------------
 * Upload a host CSR (row pointer int32[nrow+1], col int32[nnz], values of
 * val_dtype) and store it as `dtype` (cast on the way, CastFrom).  Replaces
 * Init + CopyStructureFrom + CopyFrom (lmatrix_csr_gpu.cc:135,225).  The
 * structure is validated on the host: rowptr[0] == 0, non-decreasing,
 * rowptr[nrow] == nnz, 0 <= col < ncol. */
int b200la_csr_upload(b200la_ctx ctx, int nrow, int ncol, int64_t nnz, const int *rowptr,
                      const int *col, const void *val, int val_dtype, int dtype,
                      b200la_mat *out);
/* COO -> CSR on the device: CPU_CSR_lMatrix::TransformFromCOO
 * (lmp/lmatrix_csr_cpu.cc:883-906, coo_2_csr in lmp/lmatrix_formats.h:320-452).
 * Triplets (rows[k], cols[k], val[k]) in any order, duplicates kept; the result
 * is the reference's CSR bit for bit: entries grouped by row in input order,
 * then each row sorted by column with the reference's selection sort.
 * device_input = 1: rows, cols and val are device buffers (for example from a
 * device assembler); 0: host arrays.  Every index is checked on the device; a
 * triplet out of range fails with B200LA_ERR_MATRIX.  nnz < 2^31. */
int b200la_coo_upload(b200la_ctx ctx, int nrow, int ncol, int64_t nnz, const int *rows, const int *cols,
                      const void *val, int val_dtype, int dtype, int device_input, b200la_mat *out);
/* CopyTo a host CSR (lmp/lmatrix.h CopyTo): rowptr int32[nrow+1], col
 * int32[nnz], val of the matrix's dtype [nnz], as stored. */
int b200la_mat_download(b200la_mat m, int *rowptr, int *col, void *val);
int b200la_mat_destroy(b200la_mat m);
int b200la_mat_info(b200la_mat m, int *nrow, int *ncol, int64_t *nnz, int *dtype);
/* CastFrom: a new matrix of the same structure holding the values as dtype. */
int b200la_mat_cast(b200la_mat src, int dtype, b200la_mat *out);
/* ZeroRows(index_set, size, alpha) (lmp/lmatrix_csr_cpu.cc:908-927): rows
 * become alpha*e_i, the stored pattern is kept. */
int b200la_mat_zero_rows(b200la_mat m, const int *rows, int size, double alpha);
/* VectorMult: y = A x (lmp/lmatrix.h, GPUscalar_csr_lmatrix.cu:86-107) */
int b200la_spmv(b200la_mat m, b200la_vec x, b200la_vec y);
/* VectorMultAdd: y += A x (lmatrix_csr_cpu.cc:1404-1440) */
int b200la_spmv_add(b200la_mat m, b200la_vec x, b200la_vec y);
/* VectorMultNoDiag: y = (A - diag(A)) x, every stored entry off the diagonal
 * (lmp/lmatrix_csr_cpu.cc:479-493) */
int b200la_spmv_nodiag(b200la_mat m, b200la_vec x, b200la_vec y);
/* extract_invdiagelements(0, nrow, out) (lmatrix_csr_cpu.cc:2426-2441);
 * B200LA_ERR_MATRIX if a row has no stored nonzero diagonal. */
int b200la_mat_inv_diag(b200la_mat m, b200la_vec out);
/* Pick the SpMV schedule: format B200LA_FMT_CSR with `param` threads per row
 * (1..32, power of two), or B200LA_FMT_SELL / SELL16 / STENCIL with `param`
 * entries per vector load (1, 2 or 4); builds the sliced copy on first use.
 * STENCIL (no reference counterpart): the stencil is the offsets of a
 * longest row; every row's columns must be strictly ascending and a subset
 * of it (checked on the device), and it must have 9 or 27 entries, else
 * B200LA_ERR_UNSUPPORTED.  Each row stores one value per offset (0 where it
 * has no entry; the list is padded with offset 0 to a multiple of `param`),
 * so the copy holds values only; a row's products are added in ascending
 * column order, its stored order, so the results are SELL's bits (the
 * absent entries add 0 * x at a column the row does not read: a non-finite
 * x there makes the row's sum NaN where CSR would not). */
int b200la_mat_set_format(b200la_mat m, int format, int param);
int b200la_mat_get_format(b200la_mat m, int *format, int *param);
/* SELL-C-sigma (no reference counterpart: la_global.h:56 lists an ELL format
 * the reference never implements, lmatrix_formats.h:101-110): rows sorted by
 * length, longest first, within windows of `sigma` rows (1 = rows keep their
 * order; otherwise rounded up to a multiple of C), cut into slices of C = 8,
 * 16 or 32 rows, each padded to its longest row rounded up to `width` (1, 2
 * or 4) entries per vector load; col16 = 1 stores int16 column offsets as
 * SELL16 does.  Selects the copy as the matrix's schedule (format SELL or
 * SELL16, param width).  Every variant adds each row's products in stored
 * order, so all give the same bits as SELL-32.  get_sell writes C, sigma
 * and the stored entries including padding (padded may be NULL) of the
 * current sliced schedule. */
int b200la_mat_to_sell(b200la_mat m, int C, int sigma, int width, int col16);
int b200la_mat_get_sell(b200la_mat m, int *C, int *sigma, int64_t *padded);
/* Autotuner: times every schedule on this matrix (CSR lane groups 2..32;
 * SELL and SELL16 with width 1/2/4, C = 32/16/8 and sigma 1 or 1,024;
 * STENCIL with width 1/2/4 where the matrix has a stencil; sliced copies
 * padding more than 25% skipped) and keeps the fastest.
 * Writes the chosen format/param and its time per SpMV in microseconds;
 * b200la_mat_get_sell gives the chosen C and sigma. */
int b200la_mat_tune(b200la_mat m, int *format, int *param, double *usec);

/* ---- preconditioned CG: CG<LAD> + PreconditionerBlockJacobiStand<LAD>
 * (linear_solver/cg.h:39-246, preconditioner_bjacobi_standard.cc:77-196) ---
 * The iteration is the reference's recurrence; the stopping test is
 * IterateControl::Check (common/iterate_control.cc:80-107). */
typedef struct {
  int maxits;    /* IterateControl maxits */
  double atol;   /* success if res <= atol */
  double rtol;   /* success if res < rtol * res_init */
  double dtol;   /* divergence if res > dtol * res_init */
  int precond;   /* 0: SolveNoPrecond; 1: SolvePrecond with Jacobi */
  int stop_rule; /* B200LA_STOP_ITERATE_CONTROL (0): CG<LAD> with IterateControl::Check.
                    B200LA_STOP_LMP_CG (1): the lmp cg() (lmp/solvers/cg.h:93-209,
                    cg.cc:35-41): plain CG (that function computes a preconditioned z
                    but never uses it, cg.h:153 vs :157, so precond must be 0), stop
                    after an iteration once ||r|| <= max(rtol * ||r0||, atol) (:149,
                    :193), no divergence test, at most maxits iterations; the result's
                    iters is then the 0-based index of the breaking iteration, or maxits,
                    as cg() returns it in max_iter (:201) */
} b200la_cg_params;
#define B200LA_STOP_ITERATE_CONTROL 0
#define B200LA_STOP_LMP_CG 1

typedef struct {
  int iters;        /* CG::iter_ */
  int state;        /* B200LA_ITERATE .. B200LA_FAIL_BREAKDOWN */
  int solver_state; /* B200LA_SOLVER_SUCCESS / _EXCEEDED / _ERROR */
  int reserved;
  double res;       /* CG::res_ : ||r||_2 of the recurrence residual */
  double res_init;  /* CG::res_init_ */
  double res_rel;   /* CG::res_rel_ */
} b200la_cg_result;

/* SetupOperator + (optional) SetupPreconditioner: builds the solver's
 * resident work vectors, the Jacobi inverse diagonal, and the CUDA graph that
 * runs the whole iteration on the device (no host round trip per step). */
int b200la_cg_create(b200la_mat A, const b200la_cg_params *params, b200la_cg *out);
int b200la_cg_destroy(b200la_cg s);
/* Solve(b, &x): x holds the start value on entry and the solution on exit. */
int b200la_cg_solve(b200la_cg s, b200la_vec b, b200la_vec x, b200la_cg_result *result);
/* Instrumentation: from the start value x, runs `iters` iterations as
 * separate launches with CUDA events between the kernels (same kernels as the
 * graph) and writes the mean milliseconds per launch of
 * ms[0] = SpMV + p.Ap, ms[1] = update + r.r/r.z, ms[2] = direction.
 * x is not modified. */
int b200la_cg_profile(b200la_cg s, b200la_vec b, b200la_vec x, int iters, double *ms);
/* One-shot convenience: create + solve + destroy. */
int b200la_pcg_solve(b200la_mat A, b200la_vec b, b200la_vec x, const b200la_cg_params *params,
                     b200la_cg_result *result);

/* ---- more solvers on the same kernels: the stationary Jacobi<LAD> solver /
 * smoother (linear_solver/jacobi.cc:101-356) and BiCGSTAB<LAD>
 * (linear_solver/bicgstab.h:104-473).  Like CG, each solve is one CUDA-graph
 * launch whose WHILE node runs the iteration on the device.
 *
 * Jacobi: one fused kernel per sweep computes r = b - A x_k, its norm and
 * x_{k+1} = x_k + w inv_D r (the same iterate as the reference's
 * y = inv_D (b - A_nodiag x), x = (1 - w) x + w y, rounded differently) into a
 * second buffer, so the residual test of x_k costs no extra SpMV; the test
 * runs when k is a multiple of inner_iter, as SolveNormal/SolveDamped check
 * after every inner_iter sweeps.  Smoothing modes run a fixed number of sweeps
 * (SmoothNormal: smooth_iter * inner_iter; SmoothDamped: maxits * inner_iter,
 * as jacobi.cc:276 loops to maxits_) and end in B200LA_DONE_FIXED.
 *
 * BiCGSTAB: per iteration A q with q.r0-type sums, s = r - alpha Ap, A s with
 * t.s and t.t, the x/r update with r.r and r.r0 and IterateControl, and the
 * direction update; restarts when |sigma| <= eps ||Ap|| ||r0|| and the short
 * update when ||s|| <= eps follow the reference (eps 1e-15, or 5e-16 with
 * right preconditioning).  With right Jacobi preconditioning the direction is
 * kept as q = inv_D p, so A (P p) is one SpMV of q.
 *
 * GMRES<LAD, PreLAD> (linear_solver/gmres.h:143-746), restarted after
 * size_basis steps, modified Gram-Schmidt, no or right (Jacobi)
 * preconditioning: per step one SpMV (fused with w.V_0) and one cooperative
 * kernel that runs the whole Gram-Schmidt sweep with grid barriers (every
 * wait bounded: a wait that runs out ends the solve with B200LA_ERR_TIMEOUT),
 * normalises the new basis vector and applies the Givens rotations and the
 * test; at a cycle end one pass applies x += P V y.  The basis takes
 * (size_basis + 1) vectors of device memory. */
#define B200LA_METHOD_JACOBI 1
#define B200LA_METHOD_BICGSTAB 2
#define B200LA_METHOD_GMRES 3
#define B200LA_JACOBI_SOLVE_NORMAL 0
#define B200LA_JACOBI_SOLVE_DAMPED 1
#define B200LA_JACOBI_SMOOTH_NORMAL 2
#define B200LA_JACOBI_SMOOTH_DAMPED 3
#define B200LA_DONE_FIXED 6 /* a fixed number of sweeps ran (no stopping test) */

typedef struct {
  int method;       /* B200LA_METHOD_JACOBI / _BICGSTAB */
  int maxits;       /* IterateControl maxits */
  double atol, rtol, dtol;
  int precond;      /* BiCGSTAB: 0 "NoPreconditioning", 1 "RightPreconditioning" (Jacobi) */
  int mode;         /* Jacobi SetSolveMode: B200LA_JACOBI_* */
  int inner_iter;   /* Jacobi SetInnerIter (>= 1) */
  int smooth_iter;  /* Jacobi SetNumIter (>= 1) */
  double w;         /* Jacobi SetDampingParameter (> 0; 1 in the normal modes) */
  int size_basis;   /* GMRES InitParameter(size_basis, ...): Krylov basis before a restart, 1..512 */
} b200la_solver_params;

typedef struct {
  int iters;        /* iterations (Jacobi: sweeps) */
  int state;        /* B200LA_ITERATE .. B200LA_DONE_FIXED */
  int solver_state; /* B200LA_SOLVER_SUCCESS / _EXCEEDED / _ERROR */
  int restarts;     /* BiCGSTAB restarts after the first start */
  double res;       /* ||r||_2 at the last test */
  double res_init;  /* ||r||_2 at the (last re)start */
  double res_rel;
} b200la_solver_result;

typedef struct b200la_solver_s *b200la_solver;

/* Solver objects (b200la_cg, b200la_mp, b200la_solver) keep a pointer to their
 * matrix: solve only while it lives; destroying a solver after its matrix is
 * fine (destroy touches only the context). */
int b200la_solver_create(b200la_mat A, const b200la_solver_params *params, b200la_solver *out);
int b200la_solver_destroy(b200la_solver s);
/* Solve(b, &x): x holds the start value on entry and the solution on exit. */
int b200la_solver_solve(b200la_solver s, b200la_vec b, b200la_vec x, b200la_solver_result *result);
/* Instrumentation: from the start value x, runs `passes` passes of the
 * iteration as separate launches with CUDA events between the kernels and
 * writes the mean milliseconds per launch of each kernel of a pass:
 * Jacobi ms[0] = sweep; BiCGSTAB ms[0..4] = A q, s update, A s, x/r update,
 * direction; GMRES ms[0..3] = cycle update, restart, SpMV, Arnoldi step.
 * x is not modified. */
int b200la_solver_profile(b200la_solver s, b200la_vec b, b200la_vec x, int passes, double *ms);

/* ---- Q1 system assembly on the device (no reference counterpart: the
 * reference assembles on the host through its FE stack and uploads the CSR).
 * Builds the Q1 stiffness of -div(kappa grad u) on `cells`^dim uniform cells of
 * the unit square/cube with lexicographic numbering, Dirichlet rows as
 * CoupledMatrix::diagonalize_rows leaves them (coupled_matrix.cc:452-477),
 * kappa = exp(sigma * g) per cell and RHS U[0,1) on interior rows from the
 * seed's splitmix64 streams.  Output buffers are device memory of
 * b200la_q1_size's sizes (rowptr n+1, col/val nnz, rhs n). */
int b200la_q1_size(int dim, int cells, int64_t *n, int64_t *nnz);
int b200la_q1_assemble(b200la_ctx ctx, int dim, int cells, uint64_t seed, double sigma, int *rowptr,
                       int *col, double *val, double *rhs);

/* ---- mixed-precision refinement: MPIR<LAD_high, LAD_low>::SolveImpl
 * (linear_solver/mpir.cc:52-230) with an FP32 Jacobi-PCG as the low-precision
 * error-correction solver and no smoothers.  The residual r = b - A x, the
 * update x += c and the stopping test run in FP64 on the device; the inner
 * solve runs SpMV and vector updates in FP32 (FP32 matrix values, int32
 * indices, dot products accumulated in FP32 with compensated summation).
 * The outer test is relative to the initial residual (the reference resets
 * res0_ every pass, mpir.cc:239).  By default a pass does not restart the
 * inner PCG: the FP64 residual replaces its recurrence residual and the
 * search direction carries on (restart_inner = 1 restarts it as MPIR does;
 * restarting discards the Krylov space built so far, which on the 128^3
 * lognormal case costs ~1.5x the FP64 PCG's iterations). */
typedef struct {
  int max_outer;      /* refinement passes (MPIR max_ecl) */
  double atol;        /* success if ||r||_2 <= atol */
  double rtol;        /* success if ||r||_2 < rtol * ||r0||_2 */
  double dtol;        /* divergence if ||r||_2 > dtol * ||r0||_2 */
  int inner_maxits;   /* per pass */
  double inner_rtol;  /* the FP32 solve stops at inner_rtol times its start residual */
  int precond;        /* 1: Jacobi in the FP32 solve */
  int tune;           /* 1: autotune the FP32 matrix's SpMV schedule at create */
  int inner_storage;  /* B200LA_MP_F32 (0): the inner PCG keeps FP32 vectors; B200LA_MP_F32_VALUES (1):
                         FP32 matrix values (the bulk of the bytes) under FP64 vectors, dot products
                         and Jacobi scaling */
  int restart_inner;  /* 0: every pass after the first continues the inner PCG from the new FP64
                         residual with its search direction kept (p = z + beta p, the residual
                         replacement of "reliable updates"); 1: restart it from p = z each pass, as
                         MPIR restarts its error-correction solver */
} b200la_mp_params;
#define B200LA_MP_F32 0
#define B200LA_MP_F32_VALUES 1

typedef struct {
  int outer;          /* refinement passes taken */
  int inner_iters;    /* FP32 PCG iterations over all passes */
  int state;          /* B200LA_SUCCESS_ABS/_REL, B200LA_FAIL_DIV/_MAXITS */
  int solver_state;   /* B200LA_SOLVER_SUCCESS / _EXCEEDED */
  double res;         /* final FP64 ||b - A x||_2 */
  double res_init;
  double res_rel;
} b200la_mp_result;

/* A64 must be FP64; an FP32 copy is made (CastFrom) and kept with the solver.
 * inner_storage = B200LA_MP_F32_VALUES runs the inner PCG in FP64 arithmetic
 * over that FP32 copy (each value widened before its FMA); the FP64 matrix
 * then also supplies the Jacobi inverse diagonal. */
int b200la_mp_create(b200la_mat A64, const b200la_mp_params *params, b200la_mp *out);
int b200la_mp_destroy(b200la_mp s);
/* The FP32 copy, e.g. to pick its SpMV schedule (owned by the solver). */
int b200la_mp_inner_matrix(b200la_mp s, b200la_mat *out);
/* b, x FP64; x holds the start value on entry and the solution on exit. */
int b200la_mp_solve(b200la_mp s, b200la_vec b, b200la_vec x, b200la_mp_result *result);

/* ---- batched and served PCG (no reference counterpart: the reference runs
 * one CG<LAD> solve per call).  Many independent systems of uneven size live
 * in the slots of one batch; b200la_batch_run advances every running system
 * with one CUDA-graph launch whose kernels sweep all of them, tile by tile.
 * Each system follows the Jacobi-PCG recurrence of CG<LAD>
 * (linear_solver/cg.h:165-246), either in FP64 (mixed = 0) or as FP32 inner
 * solves inside FP64 refinement (mixed = 1, MPIR structure, mpir.cc:52-230).
 * Systems can be added and removed between runs (continuous batching). */
typedef struct {
  int capacity;       /* system slots */
  int mixed;          /* 1: FP32 inner PCG + FP64 refinement; 0: FP64 PCG */
  int precond;        /* 1: Jacobi */
  int max_outer;      /* refinement passes (mixed) */
  int inner_maxits;   /* iterations per inner solve (FP64 mode: per solve) */
  int adaptive;       /* 1: each run shrinks work items (down to 32 rows) while the running
                         systems would give a kernel's warps fewer than one item each */
  int tile_rows;      /* rows per warp work item of every kernel, a multiple of 32
                         (0 = 256 SpMV, 1024 update, 512 direction; tunable) */
  int index_bits;     /* sliced-ELL column storage: 0 = no columns at all when every row's columns
                         are the row plus an ascending subset of one set of at most 27 offsets
                         (structured-grid FE couplings: values only, the column of position k
                         is row + offset k), else int16 offsets from the row when every column is
                         within int16 of its row, else int32; 16 = int16 offsets when they fit,
                         else int32; 32 = int32.  All three give the same results */
  double atol, rtol, dtol;  /* test on ||b - A x||_2 (FP64 mode: the CG recurrence residual) */
  double inner_rtol;        /* mixed: an inner pass ends at inner_rtol x its start residual */
  int restart_inner;        /* mixed: 0 = each pass continues the inner PCG from the replaced FP64
                               residual with its search direction kept (residual replacement;
                               inner_rtol ~0.1); 1 = restart it from p = z as MPIR does */
} b200la_batch_params;

typedef struct {
  int state;          /* B200LA_ITERATE while running, else the final state */
  int solver_state;   /* B200LA_SOLVER_* */
  int iters;          /* (inner) PCG iterations */
  int outer;          /* refinement passes (FP64 mode: 1) */
  int phase_done;     /* 1 once the system has finished */
  int reserved;
  double res, res_init, res_rel;  /* final FP64 residual norm, initial, ratio */
  double device_us;   /* device time from its first residual to its finish */
} b200la_sys_result;

int b200la_batch_create(b200la_ctx ctx, const b200la_batch_params *params, b200la_batch *out);
int b200la_batch_destroy(b200la_batch b);
/* Device bytes one slot holds for a system of n rows, nnz entries and
 * longest row max_row (the admission test of a request loop). */
int b200la_batch_slot_bytes(int64_t n, int64_t nnz, int max_row, int mixed, int64_t *bytes);
/* Upload one system (host CSR, FP64 values, FP64 RHS; x0 NULL = zero start)
 * into a free slot; it joins at the next run.  The structure is checked on
 * the device after the copy (the checks of b200la_csr_upload; malformed CSR
 * returns B200LA_ERR_MATRIX and leaves the slot free), so the call waits for
 * its own copies: host buffers may be reused on return. */
int b200la_batch_add(b200la_batch b, int n, int64_t nnz, const int *rowptr, const int *col,
                     const double *val, const double *rhs, const double *x0, int *slot);
/* Assemble a Q1 diffusion system on the device directly into a free slot:
 * dim 2 or 3, `cells` per axis on the unit square/cube, per-cell coefficient
 * exp(sigma * g) (sigma = 0: Poisson), homogeneous Dirichlet rows, RHS
 * U[0,1) on interior rows, from `seed` (see b200la_q1_assemble). */
int b200la_batch_add_q1(b200la_batch b, int dim, int cells, uint64_t seed, double sigma, int *slot);
/* Adds `count` systems (arrays of the arguments of b200la_batch_add; x0 may
 * be NULL, or hold NULL entries): all copies and device checks are queued,
 * then waited for once.  slots[k] is each system's slot (-1 if it failed),
 * status[k] its status; returns the first failure's status (B200LA_OK if
 * every system was added). */
int b200la_batch_add_many(b200la_batch b, int count, const int *n, const int64_t *nnz, const int *const *rowptr,
                          const int *const *col, const double *const *val, const double *const *rhs,
                          const double *const *x0, int *slots, int *status);
/* Copy a slot's system back to the host (any pointer may be NULL). */
int b200la_batch_get_system(b200la_batch b, int slot, int *rowptr, int *col, double *val, double *rhs);
int b200la_batch_slot_size(b200la_batch b, int slot, int *n, int64_t *nnz);
/* Frees a slot (stream-ordered: after the work already queued; no wait). */
int b200la_batch_remove(b200la_batch b, int slot);
/* Frees `count` slots at once (all must be in use and distinct, else nothing
 * is freed); their device states are cleared with one memset per run of
 * consecutive slots. */
int b200la_batch_remove_many(b200la_batch b, int count, const int *slots);
/* Asynchronous b200la_batch_run: enqueues one launch of at most max_passes
 * passes over the running systems and returns at once.  Systems added
 * meanwhile (b200la_batch_add* run on the batch's own transfer stream) join
 * at the next launch; the next run, solve, result(s), restart, tune or
 * profile call completes the launch first. */
int b200la_batch_launch(b200la_batch B, int max_passes);
/* One graph launch: at most max_passes iterations of every running system.
 * Writes how many systems are still running. */
int b200la_batch_run(b200la_batch b, int max_passes, int *active);
/* Registers host destinations x[k] for the solutions of slots[k]: each
 * registered system's solution is copied there as soon as a run, solve or
 * launch completion sees it finished, on the batch's transfer stream, so the
 * copies overlap the passes of the systems still running.  A later
 * b200la_batch_result(s) with the same destination only waits for the copy.
 * Destinations must stay valid until that call (pinned memory keeps the
 * copies asynchronous).  A registration ends when the slot's result is read
 * with a destination, at its removal or at a restart; x[k] = NULL cancels
 * one. */
int b200la_batch_set_outputs(b200la_batch b, int count, const int *slots, double *const *x);
/* Runs until every system has finished, in launches of at most chunk_passes
 * passes; between launches the tile list is rebuilt from the systems still
 * running.  Writes the passes taken. */
int b200la_batch_solve(b200la_batch b, int chunk_passes, int *total_passes);
/* Body passes (iterations of the device loop) taken by the last run. */
int b200la_batch_last_run(b200la_batch b, int *passes, double *reserved);
/* Result of a slot (solution copied to x if non-NULL). */
int b200la_batch_result(b200la_batch b, int slot, double *x, b200la_sys_result *result);
/* Results of `count` slots at once; x[k] (or x itself) may be NULL.  The
 * solution copies are queued together and waited for once. */
int b200la_batch_results(b200la_batch b, int count, const int *slots, double *const *x,
                         b200la_sys_result *results);
int b200la_batch_info(b200la_batch b, int *used_slots, int64_t *device_bytes);
/* Restart every system in the batch from x = 0 (matrices and RHS stay). */
int b200la_batch_restart(b200la_batch b);
/* Work is split into warp items of consecutive rows; K1 (the SpMV), K2 (the
 * update and its dot products) and K3 (the direction update) each have
 * their own item size.  set_items sets them (multiples of 32 rows; they take
 * effect at the next run); with adaptive = 1 each run halves a kernel's
 * item, down to 32 rows, while the running systems would give its warps
 * fewer than one item each (as b200la_batch_params.adaptive).  get_items
 * writes the three sizes. */
int b200la_batch_set_items(b200la_batch b, int rows_spmv, int rows_update, int rows_direction, int adaptive);
int b200la_batch_get_items(b200la_batch b, int *rows /* [3] */);
/* Autotuner: unless the batch was created with a fixed tile_rows, times
 * candidate item sizes (K1 128..256, K2/K3 256..2048 rows) on real passes
 * over the running systems, whose carried state is restored after every
 * trial, and keeps each kernel's fastest.  Writes the three item sizes and
 * the pass time (microseconds, K1 + K2 + K3). */
int b200la_batch_tune(b200la_batch b, int *rows /* [3] */, double *usec);
/* Instrumentation: mean milliseconds of the inner solve's batched SpMV over
 * every slot (reps launches, CUDA events) and its algorithmic bytes:
 * sum over systems of nnz*(value+4) + (n+1)*4 + 2*n*value. */
int b200la_batch_profile(b200la_batch b, int reps, double *ms_spmv, int64_t *algorithmic_bytes);
/* Instrumentation of the solver's own kernels: restarts every system from
 * x = 0, takes one pass, then times `reps` (1..16) inner passes kernel by
 * kernel with CUDA events -- ms[0] K1 (SpMV + p.Ap), ms[1] K2 (r update +
 * r.r, r.z), ms[2] K3 (correction c += alpha p and direction update) -- and
 * restarts again.  bytes[k] are each kernel's algorithmic bytes per launch
 * over every slot: K1 nnz*(value+4) + (n+1)*4 + 2*n*value; K2 4*n*value
 * (Jacobi) or 3; K3 6*n*value (Jacobi) or 5. */
int b200la_batch_profile_pass(b200la_batch b, int reps, double *ms, int64_t *bytes);

/* ---- request loop (no reference counterpart) ------------------------------
 * A server owns one batch and a worker thread.  Submitted solves wait in a
 * FIFO queue; between graph launches of at most chunk_passes passes the
 * worker admits queued requests first-fit while a slot is free and the
 * resident systems' device bytes (b200la_batch_slot_bytes, plus the
 * assembly's coefficient buffer for device-built requests) stay within
 * hbm_budget, then harvests finished systems: their solution and result are
 * copied to the host and the slot's memory is freed.  Admitted systems
 * share every launch with the ones already running (continuous batching);
 * matrices and Krylov state stay resident between launches.  A request the
 * queue head could not fit past is held back once the head has been passed
 * over max_skips times, so large requests are not starved.
 *
 * Threading: submit/poll/wait/stats may be called from any host thread;
 * while a server runs, its context belongs to the worker thread (make no
 * other calls on that context until b200la_server_stop returns). */
typedef struct b200la_server_s *b200la_server;

typedef struct {
  b200la_batch_params batch;  /* solver settings; batch.capacity = slots */
  int64_t hbm_budget;         /* device bytes for resident systems (0 = 90% of free memory at start) */
  int chunk_passes;           /* passes per launch between admissions and harvests (0 = 32) */
  int max_skips;              /* admission rounds the queue head may be passed over (0 = 8) */
} b200la_server_params;

typedef struct {
  int64_t submitted, completed, failed, running, queued;
  int64_t hbm_in_use, hbm_peak, hbm_budget;  /* admitted request bytes */
  int64_t launches, passes;                  /* graph launches and device passes so far */
  double p50_ms, p99_ms, mean_ms, max_ms;    /* submit-to-result latency of completed solves */
  double solves_per_s;                       /* completed / wall_s */
  double wall_s;                             /* first submission to last completion */
} b200la_server_stats;

int b200la_server_start(b200la_ctx ctx, const b200la_server_params *params, b200la_server *out);
/* Stops the worker (requests still queued or running are dropped) and frees
 * the server, its batch and every stored result. */
int b200la_server_stop(b200la_server s);
/* Queue one solve of a host CSR system (copied at submission; the caller's
 * buffers may be reused on return).  Malformed CSR returns B200LA_ERR_MATRIX
 * and a system larger than the budget B200LA_ERR_NOMEM, both at once. */
int b200la_server_submit_csr(b200la_server s, int n, int64_t nnz, const int *rowptr, const int *col,
                             const double *val, const double *rhs, const double *x0, int64_t *id);
/* Queue one solve of a Q1 diffusion system assembled on the device at
 * admission (arguments as in b200la_batch_add_q1). */
int b200la_server_submit_q1(b200la_server s, int dim, int cells, uint64_t seed, double sigma, int64_t *id);
/* done = 0 while queued or running.  Once done: the result, its latency
 * (submission to harvest, ms) and, if x is non-NULL, the solution (n
 * doubles).  A request that failed at admission returns that status. */
int b200la_server_poll(b200la_server s, int64_t id, int *done, double *x, b200la_sys_result *result,
                       double *latency_ms);
/* Blocks until request id is done or timeout_s passes (done tells which). */
int b200la_server_wait(b200la_server s, int64_t id, double timeout_s, int *done);
/* Frees a finished request's stored solution. */
int b200la_server_release(b200la_server s, int64_t id);
/* Blocks until nothing is queued or running; B200LA_ERR_TIMEOUT after timeout_s. */
int b200la_server_drain(b200la_server s, double timeout_s);
int b200la_server_get_stats(b200la_server s, b200la_server_stats *stats);
/* Clears the latency record and counters (e.g. after a warm-up stream). */
int b200la_server_reset_stats(b200la_server s);

#ifdef __cplusplus
}
#endif

#endif /* B200LA_H */
