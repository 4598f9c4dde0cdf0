// HiFlow3's own lmp code running on the B200 backend classes.
//
// Linked against the reference's lmp CPU sources compiled unmodified
// (oracle/_ref/libhiflow_lmp_ref.so: lVector/lMatrix bases, the CPU classes,
// the factories, lPreconditioner_Jacobi and the lmp cg() of
// lmp/solvers/cg.cc) and against libb200la_hiflow.so (B200_lVector,
// B200_CSR_lMatrix).  Each check prints one line "PASS <name> ..." or
// "FAIL <name> ..."; the exit status is the number of failures.
//
//   * cg_test: the reference's tests/cg_test.cc case (3x3, all 9 entries
//     stored, b = (1, -2, 0)) through the reference's cg() on B200 vectors
//     and a B200 matrix built from a CPU CSR matrix (CopyStructureFrom +
//     CopyFrom, the GPU route of the reference): x = (-0.25, -1.5, -0.75)
//     within 1e-12, the same returned iteration index as the CPU run;
//   * lmp_test: the reference's tests/lmp_test.cc SpMV (7-entry 3x3 from
//     COO, x = (1, -2, 0)) gives (4, -5, 2) through B200 VectorMult, with the
//     matrix from CopyFrom and from ConvertFrom (COO -> CSR on the device);
//   * a 2D five-point Laplacian with a variable coefficient: cg() on CPU and
//     on B200 objects, without and with lPreconditioner_Jacobi (whose Build
//     clones the B200 operator into a CPU matrix and whose Apply runs
//     CopyFrom + ElementWiseMult on B200 vectors): iteration index +-1,
//     solutions within 1e-10 relative; FP32 likewise within 1e-4;
//   * vector semantics against CPUsimple_lVector: Dot, Axpy, ScaleAdd,
//     Scale, Norm2, CastFrom/CastTo, partial_add_subvector,
//     extract_subvector, VectorMultNoDiag, extract_invdiagelements.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "lmatrix_coo_cpu.h"
#include "lmatrix_csr_cpu.h"
#include "lmp_b200.h"
#include "lpreconditioner.h"
#include "lvector_cpu.h"
#include "solvers/cg.h"

using namespace hiflow::la;

static int g_fail = 0;

static void report(bool ok, const std::string &name, const std::string &info) {
  std::printf("%s %s %s\n", ok ? "PASS" : "FAIL", name.c_str(), info.c_str());
  std::fflush(stdout);
  if (!ok) ++g_fail;
}

template < typename T > static std::vector< T > values(const lVector< T > &v) {
  std::vector< T > h(v.get_size());
  v.GetBlockValues(0, v.get_size(), h.data());
  return h;
}

template < typename T > static double rel_diff(const std::vector< T > &a, const std::vector< T > &b) {
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += ((double)a[i] - (double)b[i]) * ((double)a[i] - (double)b[i]);
    den += (double)b[i] * (double)b[i];
  }
  return std::sqrt(num / (den > 0 ? den : 1));
}

// 2D five-point operator -div(k grad u) on an m x m interior grid, k from a
// fixed smooth-but-rough formula, rows in lexicographic order
template < typename T > static void laplace(int m, CPUsimple_CSR_lMatrix< T > &A, std::vector< T > &b) {
  std::vector< int > rows, cols;
  std::vector< T > vals;
  auto kap = [&](int i, int j) { return 1.0 + 0.9 * std::sin(0.37 * i + 1.3) * std::cos(0.53 * j + 0.2); };
  const int n = m * m;
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      const int r = j * m + i;
      const double kw = 0.5 * (kap(i, j) + kap(i - 1, j)), ke = 0.5 * (kap(i, j) + kap(i + 1, j));
      const double ks = 0.5 * (kap(i, j) + kap(i, j - 1)), kn = 0.5 * (kap(i, j) + kap(i, j + 1));
      if (j > 0) rows.push_back(r), cols.push_back(r - m), vals.push_back((T)-ks);
      if (i > 0) rows.push_back(r), cols.push_back(r - 1), vals.push_back((T)-kw);
      rows.push_back(r), cols.push_back(r), vals.push_back((T)(kw + ke + ks + kn));
      if (i < m - 1) rows.push_back(r), cols.push_back(r + 1), vals.push_back((T)-ke);
      if (j < m - 1) rows.push_back(r), cols.push_back(r + m), vals.push_back((T)-kn);
    }
  A.Init((int)vals.size(), n, n, "laplace");
  A.TransformFromCOO(rows.data(), cols.data(), vals.data(), n, n, (int)vals.size());
  b.resize(n);
  for (int k = 0; k < n; ++k) b[k] = (T)(0.5 + 0.5 * std::sin(0.011 * k * k + 0.7));
}

template < typename T > static B200_CSR_lMatrix< T > *to_b200(const lMatrix< T > &cpu) {
  lMatrix< T > *m = init_matrix_b200< T >(cpu.get_nnz(), cpu.get_num_row(), cpu.get_num_col(), "A", GPU, B200, CSR);
  m->CopyStructureFrom(cpu);
  m->CopyFrom(cpu);
  return dynamic_cast< B200_CSR_lMatrix< T > * >(m);
}

static void cg_test_known_answer() {
  const int rows[9] = {0, 0, 0, 1, 1, 1, 2, 2, 2}, cols[9] = {0, 1, 2, 0, 1, 2, 0, 1, 2};
  const double vals[9] = {2, -1, 0, -1, 2, -1, 0, -1, 2};
  lMatrix< double > *Acpu = init_matrix< double >(9, 3, 3, "A", CPU, NAIVE, CSR);
  Acpu->init_structure(rows, cols);
  for (int k = 0; k < 9; ++k) Acpu->add_value(rows[k], cols[k], vals[k]);
  int it_cpu = 100, it_gpu = 100;
  std::vector< double > xc, xg;
  for (int dev = 0; dev < 2; ++dev) {
    const IMPLEMENTATION impl = dev ? B200 : NAIVE;
    const PLATFORM plat = dev ? GPU : CPU;
    lVector< double > *b = init_vector_b200< double >(3, "b", plat, impl);
    b->Zeros();
    b->add_value(0, 1.0);
    b->add_value(1, -2.0);
    b->add_value(2, 0.0);
    lVector< double > *x = init_vector_b200< double >(3, "x", plat, impl);
    x->Zeros();
    lMatrix< double > *A = dev ? (lMatrix< double > *)to_b200(*Acpu) : Acpu;
    int &it = dev ? it_gpu : it_cpu;
    const int rc = cg(x, b, A, 0.0, 0.0, it, -1);
    if (rc != 0) report(false, "cg_test", "cg() returned " + std::to_string(rc));
    (dev ? xg : xc) = values(*x);
    if (dev) delete A;
    delete x;
    delete b;
  }
  const double want[3] = {-0.25, -1.5, -0.75};
  double err = 0;
  for (int k = 0; k < 3; ++k) err = std::max(err, std::abs(xg[k] - want[k]));
  char info[256];
  std::snprintf(info, sizeof info, "x=(%.17g,%.17g,%.17g) maxerr=%.2e iters cpu=%d b200=%d", xg[0], xg[1], xg[2],
                err, it_cpu, it_gpu);
  report(err <= 1e-12 && it_cpu == it_gpu, "cg_test_known_answer", info);
  delete Acpu;
}

static void lmp_test_spmv() {
  std::vector< int > row = {0, 0, 1, 1, 1, 2, 2}, col = {0, 1, 0, 1, 2, 1, 2};
  std::vector< double > val = {2, -1, -1, 2, -1, -1, 2};
  CPUsimple_CSR_lMatrix< double > sm;
  sm.Init(7, 3, 3, "sm");
  sm.TransformFromCOO(row.data(), col.data(), val.data(), 3, 3, 7);
  CPUsimple_COO_lMatrix< double > coo;
  coo.Init(7, 3, 3, "coo");
  for (int k = 0; k < 7; ++k) {
    coo.matrix.row[k] = row[k];
    coo.matrix.col[k] = col[k];
    coo.matrix.val[k] = val[k];
  }
  B200_CSR_lMatrix< double > *A = to_b200(sm);
  B200_CSR_lMatrix< double > A2;
  A2.ConvertFrom(coo);
  for (int which = 0; which < 2; ++which) {
    B200_lVector< double > x(3, "x"), y(3, "y");
    const double xs[3] = {1.0, -2.0, 0.0};
    x.SetBlockValues(0, 3, xs);
    (which ? (lMatrix< double > &)A2 : (lMatrix< double > &)*A).VectorMult(x, &y);
    std::vector< double > h = values(y);
    char info[160];
    std::snprintf(info, sizeof info, "y=(%g,%g,%g)", h[0], h[1], h[2]);
    report(h[0] == 4.0 && h[1] == -5.0 && h[2] == 2.0, which ? "lmp_test_spmv_from_coo" : "lmp_test_spmv", info);
  }
  delete A;
}

template < typename T > static void laplace_cg(bool precond) {
  const std::string tag = std::string(sizeof(T) == 8 ? "f64" : "f32") + (precond ? "_jacobi" : "");
  CPUsimple_CSR_lMatrix< T > Acpu;
  std::vector< T > bh;
  laplace< T >(64, Acpu, bh);
  const int n = Acpu.get_num_row();
  const T rel = sizeof(T) == 8 ? (T)1e-10 : (T)1e-5;
  int iters[2] = {5000, 5000};
  std::vector< T > xs[2];
  for (int dev = 0; dev < 2; ++dev) {
    lVector< T > *b = init_vector_b200< T >(n, "b", dev ? GPU : CPU, dev ? B200 : NAIVE);
    lVector< T > *x = init_vector_b200< T >(n, "x", dev ? GPU : CPU, dev ? B200 : NAIVE);
    b->SetBlockValues(0, n, bh.data());
    x->Zeros();
    lMatrix< T > *A = dev ? (lMatrix< T > *)to_b200(Acpu) : (lMatrix< T > *)&Acpu;
    lPreconditioner_Jacobi< T > pre;
    if (precond) {
      pre.Init();
      pre.SetupOperator(*A);
      pre.Build(b, x);
    }
    cg(x, b, A, rel, (T)0, iters[dev], -1, precond ? &pre : nullptr);
    xs[dev] = values(*x);
    if (precond) pre.Clear();
    if (dev) delete A;
    delete x;
    delete b;
  }
  const double d = rel_diff(xs[1], xs[0]);
  const double tol = sizeof(T) == 8 ? 1e-10 : 1e-4;
  char info[160];
  std::snprintf(info, sizeof info, "n=%d iters cpu=%d b200=%d rel.diff=%.2e", n, iters[0], iters[1], d);
  report(std::abs(iters[0] - iters[1]) <= (sizeof(T) == 8 ? 1 : 3) && d <= tol, "laplace_cg_" + tag, info);
}

static void vector_semantics() {
  const int n = 1037;
  std::vector< double > a(n), b(n);
  for (int k = 0; k < n; ++k) {
    a[k] = std::sin(0.3 * k) + 0.01 * k;
    b[k] = std::cos(0.7 * k) - 0.5;
  }
  CPUsimple_lVector< double > ca(n, "ca"), cb(n, "cb");
  ca.SetBlockValues(0, n, a.data());
  cb.SetBlockValues(0, n, b.data());
  B200_lVector< double > ga(n, "ga"), gb(n, "gb");
  ga.CopyFrom(ca);
  gb.CopyFrom(cb);
  char info[320];
  const double dot_d = std::abs(ga.Dot(gb) - ca.Dot(cb)), nrm_d = std::abs(ga.Norm2() - ca.Norm2());
  std::snprintf(info, sizeof info, "|dot diff|=%.2e |norm diff|=%.2e", dot_d, nrm_d);
  report(dot_d <= 1e-12 * n && nrm_d <= 1e-12 * n, "vector_dot_norm2", info);
  // BLAS-1 updates: the device rounds with FMA, the CPU classes without
  ga.Axpy(gb, 0.75);
  ca.Axpy(cb, 0.75);
  ga.ScaleAdd(-1.5, gb);
  ca.ScaleAdd(-1.5, cb);
  ga.Scale(0.25);
  ca.Scale(0.25);
  const double upd = rel_diff(values(ga), values(ca));
  // partial_add_subvector / extract_subvector at unaligned offsets
  ga.partial_add_subvector(3, 5, 101, 2.0, gb);
  ca.partial_add_subvector(3, 5, 101, 2.0, cb);
  const double part = rel_diff(values(ga), values(ca));
  lVector< double > *sub = ga.extract_subvector(7, 500);
  std::vector< double > hs = values(*sub), hg = values(ga);
  bool sub_ok = (int)hs.size() == 493;
  for (int k = 0; k < 493 && sub_ok; ++k) sub_ok = hs[k] == hg[7 + k];
  delete sub;
  std::snprintf(info, sizeof info, "axpy/scaleadd/scale rel.diff=%.2e partial_add rel.diff=%.2e subvector %s", upd,
                part, sub_ok ? "exact" : "differs");
  report(upd <= 1e-15 && part <= 1e-15 && sub_ok, "vector_updates", info);
  // casts: the float copy of the device values, both directions
  B200_lVector< float > gf(n, "gf");
  gf.CastFrom(ga);
  std::vector< float > hf = values(gf);
  bool cast_ok = true;
  for (int k = 0; k < n && cast_ok; ++k) cast_ok = hf[k] == (float)hg[k];
  B200_lVector< double > gd2(n, "gd2");
  gf.CastTo(gd2);
  std::vector< double > hd2 = values(gd2);
  for (int k = 0; k < n && cast_ok; ++k) cast_ok = hd2[k] == (double)hf[k];
  report(cast_ok, "vector_casts", cast_ok ? "exact" : "differ");
  // no-diagonal product and the inverse diagonal
  CPUsimple_CSR_lMatrix< double > Acpu;
  std::vector< double > bh;
  laplace< double >(20, Acpu, bh);
  const int m = Acpu.get_num_row();
  B200_CSR_lMatrix< double > *A = to_b200(Acpu);
  CPUsimple_lVector< double > cx(m, "cx"), cy(m, "cy"), cd(m, "cd");
  cx.SetBlockValues(0, m, bh.data());
  B200_lVector< double > gx(m, "gx"), gy(m, "gy"), gd(m, "gd");
  gx.CopyFrom(cx);
  Acpu.VectorMultNoDiag(cx, &cy);
  A->VectorMultNoDiag(gx, &gy);
  Acpu.extract_invdiagelements(0, m, &cd);
  A->extract_invdiagelements(0, m, &gd);
  const double dn = rel_diff(values(gy), values(cy)), dd = rel_diff(values(gd), values(cd));
  std::snprintf(info, sizeof info, "nodiag rel.diff=%.2e invdiag rel.diff=%.2e", dn, dd);
  report(dn <= 1e-15 && dd == 0.0, "matrix_nodiag_invdiag", info);
  delete A;
}

int main() {
  cg_test_known_answer();
  lmp_test_spmv();
  laplace_cg< double >(false);
  laplace_cg< double >(true);
  laplace_cg< float >(false);
  laplace_cg< float >(true);
  vector_semantics();
  std::printf("failures %d\n", g_fail);
  return g_fail;
}
