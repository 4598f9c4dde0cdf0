// Device-side assembly of the Q1 diffusion systems on uniform grids.
//
// The reference assembles on the host through its FE stack (mesh -> dof ->
// fem -> assembly, then CoupledMatrix::diagonalize_rows for Dirichlet rows,
// linear_algebra/coupled_matrix.cc:452-477) and uploads the CSR
// (lmp/cuda/lmatrix_csr_gpu.cc:135,225).  For requests that arrive as a
// description (dimension, cells per axis, coefficient seed and sigma) the
// request loop builds the same matrix directly in the slot's HBM instead:
//   * element stiffness by Hamming distance of the two local nodes, 2D
//     [2/3, -1/6, -1/3], 3D h*[1/3, 0, -1/12, -1/12], times the sum of kappa
//     over the cells holding both nodes, summed in the same cell order as the
//     host generator (ba_b200/problems.py);
//   * Dirichlet rows keep their pattern with 1 on the diagonal, 0 elsewhere;
//   * lexicographic numbering (x fastest), columns ascending;
//   * kappa = exp(sigma * g), g by Box-Muller from two splitmix64 streams,
//     and RHS U[0,1) on interior rows from a third stream (splitmix64: Steele,
//     Lea & Flood, OOPSLA 2014).  The integer stream and the RHS are bit-equal
//     to the host generator; kappa uses the device's log/cos/exp and may
//     differ from the host's libm in the last bits.
// Row pointers are closed-form: a node's row holds prod_a L(i_a) entries with
// L(i) = 3 - [i == 0] - [i == m-1], so the entries before node (k, j, i) are
// S(k) T^2 + L(k) (S(j) T + L(j) S(i)), S(i) = sum_{t<i} L(t), T = 3m - 2.
#include <cmath>

#include "internal.cuh"

namespace b200la {

__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t stream, uint64_t i) {
  const uint64_t base = seed * 0x100000001B3ull + stream * 0x517CC1B727220A95ull;
  uint64_t z = base + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform_at(uint64_t seed, uint64_t stream, uint64_t i) {
  return (double)(splitmix_at(seed, stream, i) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void kappa_kernel(int64_t cells, uint64_t seed, double sigma, double *kappa) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += stride) {
    const double u1 = uniform_at(seed, 15, c), u2 = uniform_at(seed, 16, c);
    const double g = sqrt(-2.0 * log1p(-u1)) * cos(2.0 * 3.141592653589793 * u2);
    kappa[c] = exp(sigma * g);
  }
}

__device__ __forceinline__ int64_t axis_len(int i, int m) { return 3 - (i == 0) - (i == m - 1); }
__device__ __forceinline__ int64_t axis_before(int i) { return i == 0 ? 0 : 3 * (int64_t)i - 1; }

// One thread per node: writes the node's row pointer, columns and values,
// and its RHS entry.
template <int DIM>
__global__ void q1_kernel(int n, uint64_t seed, const double *__restrict__ kappa, int *__restrict__ rowptr,
                          int *__restrict__ col, double *__restrict__ val, double *__restrict__ b) {
  const int m = n + 1;
  const int64_t N = DIM == 2 ? (int64_t)m * m : (int64_t)m * m * m;
  const int64_t T = 3 * (int64_t)m - 2;
  const double h = 1.0 / n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < N; node += stride) {
    int idx[3] = {0, 0, 0};  // slowest axis first
    int64_t rem = node;
    for (int a = DIM - 1; a >= 0; --a) {
      idx[a] = (int)(rem % m);
      rem /= m;
    }
    int64_t before;
    if (DIM == 2) before = axis_before(idx[0]) * T + axis_len(idx[0], m) * axis_before(idx[1]);
    else
      before = axis_before(idx[0]) * T * T +
               axis_len(idx[0], m) * (axis_before(idx[1]) * T + axis_len(idx[1], m) * axis_before(idx[2]));
    rowptr[node] = (int)before;
    if (node == N - 1) rowptr[N] = (int)(DIM == 2 ? T * T : T * T * T);
    bool boundary = false;
    for (int a = 0; a < DIM; ++a) boundary |= idx[a] == 0 || idx[a] == m - 1;
    int64_t k = before;
    const int lo0 = -1, hi0 = 1;
    for (int d0 = lo0; d0 <= hi0; ++d0)
      for (int d1 = -1; d1 <= 1; ++d1)
        for (int d2 = (DIM == 3 ? -1 : 0); d2 <= (DIM == 3 ? 1 : 0); ++d2) {
          const int d[3] = {d0, d1, d2};
          bool ok = true;
          for (int a = 0; a < DIM; ++a) {
            const int v = idx[a] + d[a];
            ok &= v >= 0 && v < m;
          }
          if (!ok) continue;
          int64_t off = 0;
          for (int a = 0; a < DIM; ++a) off = off * m + d[a];
          int ham = 0;
          for (int a = 0; a < DIM; ++a) ham += d[a] != 0;
          double v;
          if (boundary) {
            v = ham == 0 ? 1.0 : 0.0;
          } else {
            // sum of kappa over the cells holding both nodes; per axis the
            // cell start is {p-1, p} (d = 0), {p} (d = +1), {p-1} (d = -1),
            // taken in the host generator's order (slowest axis outermost,
            // -1 before 0)
            double ks = 0.0;
            const int na = DIM;
            int nc[3], c0[3];
            for (int a = 0; a < na; ++a) {
              nc[a] = d[a] == 0 ? 2 : 1;
              c0[a] = d[a] == 1 ? 0 : -1;
            }
            for (int i0 = 0; i0 < nc[0]; ++i0)
              for (int i1 = 0; i1 < nc[1]; ++i1)
                for (int i2 = 0; i2 < (na == 3 ? nc[2] : 1); ++i2) {
                  const int sel[3] = {i0, i1, i2};
                  int64_t cell = 0;
                  for (int a = 0; a < na; ++a) cell = cell * n + (idx[a] + c0[a] + sel[a]);
                  ks += kappa ? kappa[cell] : 1.0;
                }
            double e;
            if (DIM == 2) e = ham == 0 ? 2.0 / 3.0 : ham == 1 ? -1.0 / 6.0 : -1.0 / 3.0;
            else e = ham == 0 ? h / 3.0 : ham == 1 ? 0.0 : -h / 12.0;
            v = e * ks;
          }
          col[k] = (int)(node + off);
          val[k] = v;
          ++k;
        }
    b[node] = boundary ? 0.0 : uniform_at(seed, 3, (uint64_t)node);
  }
}

int64_t q1_rows(int dim, int n) {
  const int64_t m = n + 1;
  return dim == 2 ? m * m : m * m * m;
}

int64_t q1_nnz(int dim, int n) {
  const int64_t t = 3 * (int64_t)n + 1;
  return dim == 2 ? t * t : t * t * t;
}

int q1_assemble(cudaStream_t st, int num_sms, int dim, int n, uint64_t seed, double sigma, int *rowptr, int *col,
                double *val, double *b) {
  B_CHECK(dim == 2 || dim == 3, B200LA_ERR_INVALID, "q1_assemble: dim %d", dim);
  B_CHECK(n >= 1, B200LA_ERR_INVALID, "q1_assemble: cells %d", n);
  B_CHECK(q1_nnz(dim, n) < (int64_t)INT32_MAX, B200LA_ERR_UNSUPPORTED, "q1_assemble: nnz exceeds int32");
  const int64_t cells = dim == 2 ? (int64_t)n * n : (int64_t)n * n * n;
  double *kappa = nullptr;
  if (sigma > 0.0) {
    B_CUDA(cudaMallocAsync(&kappa, sizeof(double) * cells, st));
    kappa_kernel<<<num_sms * 4, kBlock, 0, st>>>(cells, seed, sigma, kappa);
    B_CUDA(cudaGetLastError());
  }
  if (dim == 2) q1_kernel<2><<<num_sms * 4, kBlock, 0, st>>>(n, seed, kappa, rowptr, col, val, b);
  else q1_kernel<3><<<num_sms * 4, kBlock, 0, st>>>(n, seed, kappa, rowptr, col, val, b);
  B_CUDA(cudaGetLastError());
  if (kappa) B_CUDA(cudaFreeAsync(kappa, st));
  return B200LA_OK;
}

}  // namespace b200la

using namespace b200la;

extern "C" int b200la_q1_size(int dim, int cells, int64_t *n, int64_t *nnz) {
  B_CHECK((dim == 2 || dim == 3) && cells >= 1 && n && nnz, B200LA_ERR_INVALID, "q1_size: bad argument");
  *n = q1_rows(dim, cells);
  *nnz = q1_nnz(dim, cells);
  return B200LA_OK;
}

extern "C" int b200la_q1_assemble(b200la_ctx ctx, int dim, int cells, uint64_t seed, double sigma, int *rowptr,
                                  int *col, double *val, double *rhs) {
  B_CHECK(ctx && rowptr && col && val && rhs, B200LA_ERR_INVALID, "q1_assemble: null argument");
  return q1_assemble(ctx->stream, ctx->num_sms, dim, cells, seed, sigma, rowptr, col, val, rhs);
}
