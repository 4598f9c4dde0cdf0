// C++ host layer test (ba_b200/host/b200_lmp.hpp) through the C ABI, written
// like the reference's Boost tests: tests/lmp_test.cc (CSR SpMV known answer),
// tests/cuda_test.cc (GPU SpMV known answer), tests/cg_test.cc (CG known
// answer), plus a 2D Q1 Poisson Jacobi-PCG checked against the CPU oracle
// (oracle/liboracle.so, test infrastructure), the mixed-precision solver,
// Jacobi/BiCGSTAB/GMRES on the CG known answer and a generic MPIR.
#include <cmath>
#include <cstdio>
#include <vector>

#include "b200_lmp.hpp"

extern "C" int orc_cg_d(int n, const int *rowptr, const int *col, const double *val, const double *b,
                        double *x, int maxits, double atol, double rtol, double dtol, int precond,
                        const double *invd, double *work, int *iters, double *res, double *res_init);
extern "C" int orc_invdiag_d(int n, const int *rowptr, const int *col, const double *val, double *invd);

static int failures = 0;
#define CHECK(cond)                                                  \
  do {                                                               \
    if (!(cond)) {                                                   \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);  \
      ++failures;                                                    \
    }                                                                \
  } while (0)

using namespace b200la;

// 2D Q1 Poisson, n x n cells, Dirichlet identity rows with full pattern.
static void poisson2d(int n, std::vector<int> &rp, std::vector<int> &cl, std::vector<double> &va,
                      std::vector<double> &b) {
  const int m = n + 1;
  rp.assign(1, 0);
  cl.clear();
  va.clear();
  b.assign(m * m, 0.0);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      const int row = j * m + i;
      const bool bnd = i == 0 || j == 0 || i == m - 1 || j == m - 1;
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          const int ii = i + di, jj = j + dj;
          if (ii < 0 || jj < 0 || ii >= m || jj >= m) continue;
          const int ham = (di != 0) + (dj != 0);
          double v = ham == 0 ? 8.0 / 3.0 : -1.0 / 3.0;
          if (bnd) v = ham == 0 ? 1.0 : 0.0;
          cl.push_back(jj * m + ii);
          va.push_back(v);
        }
      rp.push_back((int)cl.size());
      if (!bnd) b[row] = 0.25 + 0.5 * std::sin(0.37 * row);
    }
}

int main() {
  Platform plat(0);
  {  // lmp_test.cc:42-89: 7-nnz CSR times (1,-2,0) = (4,-5,2)
    int rp[] = {0, 2, 5, 7}, cl[] = {0, 1, 0, 1, 2, 1, 2};
    double va[] = {2, -1, -1, 2, -1, -1, 2}, xin[] = {1, -2, 0}, y[3];
    B200_CSR_lMatrix<double> A(plat, 3, 3, 7, rp, cl, va);
    B200_lVector<double> x(plat, 3), out(plat, 3);
    x.SetBlockValues(0, 3, xin);
    A.VectorMult(x, &out);
    out.GetBlockValues(0, 3, y);
    CHECK(y[0] == 4.0 && y[1] == -5.0 && y[2] == 2.0);
  }
  int rp9[] = {0, 3, 6, 9}, cl9[] = {0, 1, 2, 0, 1, 2, 0, 1, 2};
  double va9[] = {2, -1, 0, -1, 2, -1, 0, -1, 2};
  {  // cuda_test.cc:38-78: dense-stored 3x3 times (1.2,-2.3,0.7) = (4.7,-6.5,3.7)
    double xin[] = {1.2, -2.3, 0.7}, y[3];
    B200_CSR_lMatrix<double> A(plat, 3, 3, 9, rp9, cl9, va9);
    B200_lVector<double> x(plat, 3), out(plat, 3);
    x.SetBlockValues(0, 3, xin);
    A.VectorMult(x, &out);
    out.GetBlockValues(0, 3, y);
    CHECK(std::fabs(y[0] - 4.7) < 1e-12 && std::fabs(y[1] + 6.5) < 1e-12 && std::fabs(y[2] - 3.7) < 1e-12);
  }
  {  // cg_test.cc:44-94: x = (-0.25, -1.5, -0.75)
    double bin[] = {1, -2, 0}, zero[] = {0, 0, 0}, xs[3];
    B200_CSR_lMatrix<double> A(plat, 3, 3, 9, rp9, cl9, va9);
    B200_lVector<double> b(plat, 3), x(plat, 3);
    b.SetBlockValues(0, 3, bin);
    for (int pc = 0; pc < 2; ++pc) {
      x.SetBlockValues(0, 3, zero);
      B200_CG<double> cg;
      cg.InitControl(100, 0.0, 1e-14, 1e8);
      cg.SetupOperator(A);
      if (pc) cg.SetupPreconditionerJacobi();
      CHECK(cg.Solve(b, &x) == kSolverSuccess);
      x.GetBlockValues(0, 3, xs);
      CHECK(std::fabs(xs[0] + 0.25) < 1e-12 && std::fabs(xs[1] + 1.5) < 1e-12 && std::fabs(xs[2] + 0.75) < 1e-12);
    }
  }
  {  // 2D Q1 Poisson 64^2: Jacobi-PCG iterations and solution vs the oracle
    std::vector<int> rp, cl;
    std::vector<double> va, bh;
    poisson2d(64, rp, cl, va, bh);
    const int n = (int)bh.size();
    B200_CSR_lMatrix<double> A(plat, n, n, (int64_t)cl.size(), rp.data(), cl.data(), va.data());
    A.Tune();
    B200_lVector<double> b(plat, n), x(plat, n);
    b.SetBlockValues(0, n, bh.data());
    x.Zeros();
    B200_CG<double> cg;
    cg.InitControl(10000, 0.0, 1e-10, 1e8);
    cg.SetupOperator(A);
    cg.SetupPreconditionerJacobi();
    CHECK(cg.Solve(b, &x) == kSolverSuccess);
    std::vector<double> xg(n), xo(n, 0.0), invd(n), work(5 * (size_t)n);
    x.GetBlockValues(0, n, xg.data());
    orc_invdiag_d(n, rp.data(), cl.data(), va.data(), invd.data());
    int it = 0;
    double res = 0, res0 = 0;
    orc_cg_d(n, rp.data(), cl.data(), va.data(), bh.data(), xo.data(), 10000, 0.0, 1e-10, 1e8, 1, invd.data(),
             work.data(), &it, &res, &res0);
    CHECK(std::abs(cg.iter() - it) <= 1);
    double num = 0, den = 0;
    for (int i = 0; i < n; ++i) {
      num += (xg[i] - xo[i]) * (xg[i] - xo[i]);
      den += xo[i] * xo[i];
    }
    CHECK(std::sqrt(num) <= 1e-10 * std::sqrt(den));
    std::printf("poisson2d_64: gpu iters %d oracle iters %d rel.diff %.2e\n", cg.iter(), it, std::sqrt(num / den));
    // mixed precision to 1e-10 relative FP64 residual
    B200_lVector<double> xm(plat, n);
    xm.Zeros();
    B200_MPIR mp(plat);
    mp.SetupOperator(A);
    mp.SetMpirParameters(0, 20, 0.0, 1e-10, 1e6);
    mp.SetLowPrecErrCorSolverParameters(100000, 0.f, 1e-5f, 1e30f);
    CHECK(mp.Solve(b, &xm) == kSolverSuccess);
    CHECK(mp.res_rel() < 1e-10);
    std::printf("mpir: outer %d inner iters %d res_rel %.2e\n", mp.outer(), mp.iter(), mp.res_rel());
  }
  {  // Jacobi, BiCGSTAB and GMRES on the cg_test.cc system: x = (-0.25, -1.5, -0.75)
    double bin[] = {1, -2, 0}, zero[] = {0, 0, 0}, xs[3];
    B200_CSR_lMatrix<double> A(plat, 3, 3, 9, rp9, cl9, va9);
    B200_lVector<double> b(plat, 3), x(plat, 3);
    b.SetBlockValues(0, 3, bin);
    B200_Jacobi<double> jac;
    B200_BiCGSTAB<double> bicg;
    bicg.InitParameter("RightPreconditioning");
    B200_GMRES<double> gm;
    gm.InitParameter(3, "RightPreconditioning");
    B200_LinearSolver<double> *solvers[] = {&jac, &bicg, &gm};
    for (B200_LinearSolver<double> *s : solvers) {
      x.SetBlockValues(0, 3, zero);
      s->InitControl(5000, 0.0, 1e-15, 1e8);
      s->SetupOperator(A);
      CHECK(s->Solve(b, &x) == kSolverSuccess);
      x.GetBlockValues(0, 3, xs);
      CHECK(std::fabs(xs[0] + 0.25) < 1e-12 && std::fabs(xs[1] + 1.5) < 1e-12 && std::fabs(xs[2] + 0.75) < 1e-12);
    }
  }
  {  // generic MPIR: FP32 GMRES error correction with FP32 Jacobi smoothing,
     // FP64 BiCGSTAB correction once the low passes are spent
    std::vector<int> rp, cl;
    std::vector<double> va, bh;
    poisson2d(48, rp, cl, va, bh);
    const int n = (int)bh.size();
    B200_CSR_lMatrix<double> A(plat, n, n, (int64_t)cl.size(), rp.data(), cl.data(), va.data());
    B200_lVector<double> b(plat, n), x(plat, n);
    b.SetBlockValues(0, n, bh.data());
    x.Zeros();
    B200_GMRES<float> ecl;
    ecl.InitParameter(30, "RightPreconditioning");
    B200_Jacobi<float> smooth;
    smooth.SetSolveMode(2);
    smooth.SetNumIter(3);
    B200_BiCGSTAB<double> ech;
    ech.InitParameter("RightPreconditioning");
    B200_MPIR mp(plat);
    mp.SetupOperator(A);
    mp.SetLowPrecErrCorSolver(ecl);
    mp.SetHighPrecErrCorSolver(ech);
    mp.SetLowPrecPreSmoother(smooth);
    mp.UseLowPrecPreSmoother(true);
    mp.SetMpirParameters(2, 2, 1e-9, 1e-14, 1e8);
    mp.SetLowPrecErrCorSolverParameters(2000, 0.0, 1e-4, 1e8);
    mp.SetLowPrecPreSmootherParameters(3, 0.0, 0.0, 1e8);
    mp.SetHighPrecErrCorSolverParameters(2000, 1e-12, 1e-6, 1e8);
    CHECK(mp.Solve(b, &x) == kSolverSuccess);
    CHECK(mp.n_ecl() == 2 && mp.n_ech() >= 1);
    std::vector<double> xg(n), r(n);
    x.GetBlockValues(0, n, xg.data());
    double rr = 0, bb = 0;
    for (int i = 0; i < n; ++i) {
      double y = 0;
      for (int k = rp[i]; k < rp[i + 1]; ++k) y += va[k] * xg[cl[k]];
      rr += (bh[i] - y) * (bh[i] - y);
      bb += bh[i] * bh[i];
    }
    CHECK(std::sqrt(rr) <= 1e-9 * 1.001);
    std::printf("generic mpir: passes %d (low %d, high %d) iters %d res %.2e\n", mp.outer(), mp.n_ecl(), mp.n_ech(),
                mp.iter(), mp.res());
  }
  {  // errors are reported, not exit(-1)
    int rp2[] = {0, 2, 1};
    int cl2[] = {0, 1};
    double va2[] = {1, 1};
    bool threw = false;
    try {
      B200_CSR_lMatrix<double> bad(plat, 2, 2, 2, rp2, cl2, va2);
    } catch (const Error &e) {
      threw = e.status == B200LA_ERR_MATRIX;
    }
    CHECK(threw);
  }
  std::printf(failures ? "FAILED (%d)\n" : "OK\n", failures);
  return failures ? 1 : 0;
}
