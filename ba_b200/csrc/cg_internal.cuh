// Solver state shared by the CG translation unit (pcg.cu) and the solvers
// built on it (mixed-precision refinement in mp.cu).
#pragma once

#include "internal.cuh"

namespace b200la {

constexpr int kMaxIts = 10000000;

// Device-resident scalars of one CG solve.
struct CgScalars {
  double rz;        // r.z of the current residual (r.r without preconditioner)
  double rz_prev;   // r.z before the last step (the denominator of the next beta)
  double pAp;
  double alpha;
  double beta;
  double rr;
  double res;
  double res_init;
  double atol, rtol, dtol;
  int iter;
  int state;
  int maxits;
  int guard;        // body passes, counted by the direction kernel
  int stop_rule;    // B200LA_STOP_ITERATE_CONTROL or B200LA_STOP_LMP_CG
  unsigned ticket[4];
};

}  // namespace b200la

struct b200la_cg_s {
  b200la_mat A;
  b200la_ctx ctx;              // kept for destroy, which may come after A's
  b200la_cg_params prm;
  int vdtype;                  // type of the work vectors and scalars' arithmetic: A's own, or FP64
                               // over an FP32 matrix (mixed storage)
  int64_t n;
  void *x, *r, *p, *Ap, *invd;
  double *part;                // [2][kMaxReduceBlocks]
  b200la::CgScalars *sc;       // device
  b200la::CgScalars *sc_host;  // pinned
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int g_format, g_param;       // schedule baked into the graph
  int g_gen;                   // the matrix's schedule generation at capture
  int grid_spmv, grid_ew;
};

namespace b200la {

// Creates a CG solver whose work vectors have type vdtype: A->dtype (as
// b200la_cg_create), or FP64 over an FP32 matrix, whose values are then
// widened to FP64 in the SpMV; the Jacobi inverse diagonal then comes from
// invd_src (an FP64 matrix of A's structure).
int cg_create_ex(b200la_mat A, const b200la_cg_params *prm, int vdtype, b200la_mat invd_src, b200la_cg *out);

// Start a solve on the context stream: r = b - A x0 (x0, b device buffers of
// the solver's value type), or r = b with x0 = 0 when x_dev is nullptr.
int cg_start(b200la_cg s, const void *x_dev, const void *b_dev);
// Continue a solve from a new residual already written to s->r (an outer
// refinement pass replaced the recurrence residual by the true one): x = 0,
// z = invD r, and p = z + beta p with beta = rz_new / rz_prev (the search
// direction is kept), or p = z when `restart`.  sums = {r.r, r.z} of the new
// residual (device; r.r twice without preconditioner).
int cg_resume(b200la_cg s, const double *sums, bool restart);
// Run the device loop (one graph launch); the solution stays in s->x.
int cg_run(b200la_cg s);
// Copy the scalars to the host (synchronises the context stream).
int cg_fetch(b200la_cg s, CgScalars *out);

}  // namespace b200la
