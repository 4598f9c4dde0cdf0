/*
 * b200la -- B200-native (sm_100a) local linear algebra for HiFlow3's
 * Jacobi-preconditioned CG hot path.  C ABI: opaque handles, plain pointers
 * and sizes, int status codes (0 = ok, < 0 = error, never exit()).
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the HiFlow3 source tree, src/).  A reference binding
 * registers these behind lmp's lVector / lMatrix / lPreconditioner and the
 * linear_solver CG interface; see INTEGRATION.md.
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
#define B200LA_FMT_SELL 4 /* SELL-C-sigma, C = 32 rows per slice */

/* ---- library / context ---------------------------------------------------
 * replaces init_platform_gpu (lmp/cuda/platform_management_gpu.cu:78-143) */
const char *b200la_version(void);
const char *b200la_last_error(void); /* message of this thread's last error */
int b200la_ctx_create(int device, b200la_ctx *out);
int b200la_ctx_destroy(b200la_ctx ctx);
/* Use an external cudaStream_t (NULL: the context's own stream). */
int b200la_ctx_set_stream(b200la_ctx ctx, void *stream);
int b200la_ctx_get_stream(b200la_ctx ctx, void **stream);
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
 * is rejected with B200LA_ERR_UNSUPPORTED.  The first call on a device looks
 * up the array's device address and caches it; make that first call before
 * any stream capture.  All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller. */
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
/* extract_invdiagelements(0, nrow, out) (lmatrix_csr_cpu.cc:2426-2441);
 * B200LA_ERR_MATRIX if a row has no stored nonzero diagonal. */
int b200la_mat_inv_diag(b200la_mat m, b200la_vec out);
/* Pick the SpMV schedule: format B200LA_FMT_CSR with `param` threads per row
 * (1..32, power of two), or B200LA_FMT_SELL with `param` rows per thread
 * chunk width (1, 2 or 4); builds the SELL copy on first use. */
int b200la_mat_set_format(b200la_mat m, int format, int param);
int b200la_mat_get_format(b200la_mat m, int *format, int *param);
/* Autotuner: times every schedule on this matrix and keeps the fastest.
 * Writes the chosen format/param and its time per SpMV in microseconds. */
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
} b200la_cg_params;

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

#ifdef __cplusplus
}
#endif

#endif /* B200LA_H */
