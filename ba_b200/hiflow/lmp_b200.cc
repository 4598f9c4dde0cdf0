// HiFlow3 lmp backend on B200: B200_lVector<T> and B200_CSR_lMatrix<T> over
// the b200la C ABI (see lmp_b200.h).  Compiled against HiFlow3's lmp headers,
// instantiated for double and float like the lmp classes themselves.
#include "lmp_b200.h"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <mutex>

#include "lmatrix_coo_cpu.h"
#include "lmatrix_csr_cpu.h"
#include "lvector_cpu.h"

namespace hiflow {
namespace la {

namespace {

std::mutex g_ctx_mu;
b200la_ctx g_ctx = nullptr;
int g_device = 0;

// HiFlow3's error convention: log and terminate (lmp/cuda/cuda_utils.h:24-55).
void fail(const char *where, const char *what) {
  LOG_ERROR(where << ": " << what);
  std::cerr << "Information: Program was terminated. " << __FILE__ << ", " << __LINE__ << "." << std::endl;
  exit(-1);
}

void check(int rc, const char *where) {
  if (rc != B200LA_OK) fail(where, b200la_last_error());
}

template < typename T > constexpr int dtype_of();
template <> constexpr int dtype_of< double >() { return B200LA_F64; }
template <> constexpr int dtype_of< float >() { return B200LA_F32; }

template < typename T > const B200_lVector< T > *as_b200(const lVector< T > &v) {
  return dynamic_cast< const B200_lVector< T > * >(&v);
}

template < typename T > b200la_vec need_b200(const lVector< T > &v, const char *where) {
  const B200_lVector< T > *b = as_b200(v);
  if (!b) fail(where, "the other vector is not a B200 vector of the same value type");
  return b->handle();
}

} // namespace

void b200_lmp_set_device(int device) {
  std::lock_guard< std::mutex > lock(g_ctx_mu);
  if (g_ctx) fail("b200_lmp_set_device", "the B200 context already exists");
  g_device = device;
}

b200la_ctx b200_lmp_context() {
  std::lock_guard< std::mutex > lock(g_ctx_mu);
  if (!g_ctx) check(b200la_ctx_create(g_device, &g_ctx), "b200_lmp_context");
  return g_ctx;
}

// ---------------------------------------------------------------- vectors

template < typename T > B200_lVector< T >::B200_lVector() {
  this->platform_name_ = "GPU (B200)";
  this->platform_id_ = GPU;
  this->implementation_name_ = "B200 (sm_100a)";
  this->implementation_id_ = B200;
  this->size_ = 0;
}

template < typename T > B200_lVector< T >::B200_lVector(int size, const std::string &name) : B200_lVector() {
  this->Init(size, name);
}

template < typename T > B200_lVector< T >::~B200_lVector() { this->Clear(); }

template < typename T > void B200_lVector< T >::Init(const int size, const std::string name) {
  this->Clear();
  check(b200la_vec_create(b200_lmp_context(), size, dtype_of< T >(), &vec_), "B200_lVector::Init");
  this->size_ = size;
  this->name_ = name;
}

template < typename T > void B200_lVector< T >::Clear(void) {
  if (vec_) b200la_vec_destroy(vec_);
  vec_ = nullptr;
  this->size_ = 0;
  indexset_.clear();
}

template < typename T > void B200_lVector< T >::Zeros(void) {
  if (this->size_ > 0) check(b200la_vec_zeros(vec_), "B200_lVector::Zeros");
}

template < typename T > std::vector< T > B200_lVector< T >::download() const {
  std::vector< T > h(this->size_);
  if (this->size_ > 0) check(b200la_vec_download(vec_, h.data(), this->size_), "B200_lVector download");
  return h;
}

template < typename T > void B200_lVector< T >::upload(const std::vector< T > &h) {
  if (this->size_ > 0) check(b200la_vec_upload(vec_, h.data(), this->size_), "B200_lVector upload");
}

template < typename T > void B200_lVector< T >::add_value(const int i, T val) {
  assert(i >= 0 && i < this->size_);
  T v = this->GetValue(i);
  v += val;
  this->SetValue(i, v);
}

template < typename T > void B200_lVector< T >::add_values(const int *indices, int length, const T *values) {
  std::vector< T > cur(length);
  this->GetValues(indices, length, cur.data());
  for (int k = 0; k < length; ++k) cur[k] += values[k];
  this->SetValues(indices, length, cur.data());
}

template < typename T > void B200_lVector< T >::SetValues(const int *index, const int size, const T *values) {
  if (size > 0) check(b200la_vec_set_values(vec_, index, values, size), "B200_lVector::SetValues");
}

template < typename T > void B200_lVector< T >::SetValue(const int index, const T value) {
  this->SetValues(&index, 1, &value);
}

template < typename T > void B200_lVector< T >::GetValues(const int *index, const int size, T *values) const {
  if (size > 0) check(b200la_vec_get_values(vec_, index, values, size), "B200_lVector::GetValues");
}

template < typename T > T B200_lVector< T >::GetValue(const int index) const {
  T v = T(0);
  this->GetValues(&index, 1, &v);
  return v;
}

template < typename T > void B200_lVector< T >::SetBlockValues(const int start_i, const int end_i, const T *values) {
  assert(start_i >= 0 && start_i <= end_i && end_i <= this->size_);
  std::vector< int > idx(end_i - start_i);
  for (int k = 0; k < end_i - start_i; ++k) idx[k] = start_i + k;
  this->SetValues(idx.data(), (int)idx.size(), values);
}

template < typename T > void B200_lVector< T >::GetBlockValues(const int start_i, const int end_i, T *values) const {
  assert(start_i >= 0 && start_i <= end_i && end_i <= this->size_);
  std::vector< int > idx(end_i - start_i);
  for (int k = 0; k < end_i - start_i; ++k) idx[k] = start_i + k;
  this->GetValues(idx.data(), (int)idx.size(), values);
}

template < typename T > void B200_lVector< T >::set_indexset(const int *indexset, const int size) {
  indexset_.assign(indexset, indexset + size);
}

template < typename T > void B200_lVector< T >::get_indexset(int *indexset) const {
  std::copy(indexset_.begin(), indexset_.end(), indexset);
}

template < typename T > int B200_lVector< T >::get_indexset_size(void) const { return (int)indexset_.size(); }

template < typename T > void B200_lVector< T >::GetIndexedValues(T *values) const {
  this->GetValues(indexset_.data(), (int)indexset_.size(), values);
}

template < typename T > void B200_lVector< T >::SetIndexedValues(const T *values) {
  this->SetValues(indexset_.data(), (int)indexset_.size(), values);
}

template < typename T > lVector< T > *B200_lVector< T >::extract_subvector(const int start_i, const int end_i) const {
  assert(start_i >= 0 && start_i <= end_i && end_i <= this->size_);
  B200_lVector< T > *sub = new B200_lVector< T >(end_i - start_i, "sub vector of " + this->name_);
  check(b200la_vec_range_update(sub->handle(), 0, vec_, start_i, end_i - start_i, 0, 0.0),
        "B200_lVector::extract_subvector");
  return sub;
}

template < typename T >
void B200_lVector< T >::partial_replace_subvector(const int start_i, const int start_sub_vec, const int size,
                                                  const lVector< T > &sub_vec) {
  check(b200la_vec_range_update(vec_, start_i, need_b200(sub_vec, "B200_lVector::partial_replace_subvector"),
                                start_sub_vec, size, 0, 0.0),
        "B200_lVector::partial_replace_subvector");
}

template < typename T >
void B200_lVector< T >::partial_add_subvector(const int start_i, const int start_sub_vec, const int size,
                                              const T weight, const lVector< T > &sub_vec) {
  check(b200la_vec_range_update(vec_, start_i, need_b200(sub_vec, "B200_lVector::partial_add_subvector"),
                                start_sub_vec, size, 1, (double)weight),
        "B200_lVector::partial_add_subvector");
}

template < typename T > void B200_lVector< T >::Reorder(const int *index) {
  // new[i] = old[index[i]], as CPU_lVector::Reorder (lmp/lvector_cpu.cc)
  std::vector< T > h = download(), r(this->size_);
  for (int i = 0; i < this->size_; ++i) r[i] = h[index[i]];
  upload(r);
}

template < typename T > lVector< T > &B200_lVector< T >::operator=(const lVector< T > &vec2) {
  if (this != &vec2) this->CopyFrom(vec2);
  return *this;
}

template < typename T > void B200_lVector< T >::CopyFrom(const lVector< T > &vec) {
  if (this == &vec) return;
  assert(this->size_ == vec.get_size());
  if (const B200_lVector< T > *b = as_b200(vec)) {
    check(b200la_vec_copy(vec_, b->handle()), "B200_lVector::CopyFrom");
  } else if (const CPU_lVector< T > *c = dynamic_cast< const CPU_lVector< T > * >(&vec)) {
    if (this->size_ > 0) check(b200la_vec_upload(vec_, c->buffer, this->size_), "B200_lVector::CopyFrom");
  } else {
    vec.CopyTo(*this);
  }
}

template < typename T > void B200_lVector< T >::CopyTo(lVector< T > &vec) const {
  if (this == &vec) return;
  assert(this->size_ == vec.get_size());
  if (B200_lVector< T > *b = dynamic_cast< B200_lVector< T > * >(&vec)) {
    check(b200la_vec_copy(b->handle(), vec_), "B200_lVector::CopyTo");
  } else if (CPU_lVector< T > *c = dynamic_cast< CPU_lVector< T > * >(&vec)) {
    if (this->size_ > 0) check(b200la_vec_download(vec_, c->buffer, this->size_), "B200_lVector::CopyTo");
  } else {
    vec.CopyFrom(*this);
  }
}

namespace {
// this <- other with a cast: B200 -> B200 on the device, CPU -> B200 on the
// host, anything else through the other side's CastTo
template < typename T, typename S > void cast_into(B200_lVector< T > &dst, const lVector< S > &src) {
  assert(dst.get_size() == src.get_size());
  if (const B200_lVector< S > *b = dynamic_cast< const B200_lVector< S > * >(&src)) {
    check(b200la_vec_cast(dst.handle(), b->handle()), "B200_lVector::CastFrom");
  } else if (const CPU_lVector< S > *c = dynamic_cast< const CPU_lVector< S > * >(&src)) {
    std::vector< T > h(dst.get_size());
    for (int i = 0; i < dst.get_size(); ++i) h[i] = (T)c->buffer[i];
    if (!h.empty()) check(b200la_vec_upload(dst.handle(), h.data(), h.size()), "B200_lVector::CastFrom");
  } else {
    src.CastTo(dst);
  }
}

template < typename T, typename S > void cast_from(const B200_lVector< T > &src, lVector< S > &dst) {
  assert(dst.get_size() == src.get_size());
  if (B200_lVector< S > *b = dynamic_cast< B200_lVector< S > * >(&dst)) {
    check(b200la_vec_cast(b->handle(), src.handle()), "B200_lVector::CastTo");
  } else if (CPU_lVector< S > *c = dynamic_cast< CPU_lVector< S > * >(&dst)) {
    std::vector< T > h(src.get_size());
    if (!h.empty()) check(b200la_vec_download(src.handle(), h.data(), h.size()), "B200_lVector::CastTo");
    for (int i = 0; i < src.get_size(); ++i) c->buffer[i] = (S)h[i];
  } else {
    dst.CastFrom(src);
  }
}
} // namespace

template < typename T > void B200_lVector< T >::CastFrom(const lVector< double > &vec) { cast_into(*this, vec); }
template < typename T > void B200_lVector< T >::CastFrom(const lVector< float > &vec) { cast_into(*this, vec); }
template < typename T > void B200_lVector< T >::CastTo(lVector< double > &vec) const { cast_from(*this, vec); }
template < typename T > void B200_lVector< T >::CastTo(lVector< float > &vec) const { cast_from(*this, vec); }

template < typename T > lVector< T > *B200_lVector< T >::CloneWithoutContent(void) const {
  // lVector::CloneWithoutContent (lmp/lvector.cc:47-57) goes through
  // init_vector, which HiFlow3 extends with the B200 case; the clone is
  // made here directly
  return new B200_lVector< T >(this->size_, "clone from " + this->name_);
}

template < typename T > void B200_lVector< T >::Sync(void) const {
  check(b200la_ctx_synchronize(b200_lmp_context()), "B200_lVector::Sync");
}

template < typename T > void B200_lVector< T >::ElementWiseMult(const lVector< T > &vec) const {
  check(b200la_vec_elementwise_mult(vec_, need_b200(vec, "B200_lVector::ElementWiseMult")),
        "B200_lVector::ElementWiseMult");
}

// ArgMin/ArgMax (first index of the smallest/largest |x_i|, as BLAS i?amin /
// i?amax), Norm1, NormMax and ContainsNaN read the vector back to the host:
// they are diagnostics, not on the solver path.
template < typename T > int B200_lVector< T >::ArgMin(void) const {
  std::vector< T > h = download();
  int k = 0;
  for (int i = 1; i < (int)h.size(); ++i)
    if (std::abs(h[i]) < std::abs(h[k])) k = i;
  return k;
}

template < typename T > int B200_lVector< T >::ArgMax(void) const {
  std::vector< T > h = download();
  int k = 0;
  for (int i = 1; i < (int)h.size(); ++i)
    if (std::abs(h[i]) > std::abs(h[k])) k = i;
  return k;
}

template < typename T > T B200_lVector< T >::Norm1(void) const {
  std::vector< T > h = download();
  T s = T(0);
  for (T v : h) s += std::abs(v);
  return s;
}

template < typename T > T B200_lVector< T >::NormMax(void) const {
  std::vector< T > h = download();
  T s = T(0);
  for (T v : h) s = std::max(s, std::abs(v));
  return s;
}

template < typename T > bool B200_lVector< T >::ContainsNaN() const {
  std::vector< T > h = download();
  for (T v : h)
    if (v != v) return true;
  return false;
}

template < typename T > T B200_lVector< T >::Norm2(void) const {
  double r = 0.0;
  if (this->size_ > 0) check(b200la_vec_norm2(vec_, &r), "B200_lVector::Norm2");
  return (T)r;
}

template < typename T > T B200_lVector< T >::Dot(const lVector< T > &vec) const {
  double r = 0.0;
  if (this->size_ > 0) check(b200la_vec_dot(vec_, need_b200(vec, "B200_lVector::Dot"), &r), "B200_lVector::Dot");
  return (T)r;
}

template < typename T > void B200_lVector< T >::Scale(const T scalar) {
  if (this->size_ > 0) check(b200la_vec_scale(vec_, (double)scalar), "B200_lVector::Scale");
}

template < typename T > void B200_lVector< T >::Axpy(const lVector< T > &vec, const T scalar) {
  if (this->size_ > 0)
    check(b200la_vec_axpy(vec_, need_b200(vec, "B200_lVector::Axpy"), (double)scalar), "B200_lVector::Axpy");
}

template < typename T > void B200_lVector< T >::ScaleAdd(const T scalar, const lVector< T > &vec) {
  if (this->size_ > 0)
    check(b200la_vec_scaleadd(vec_, (double)scalar, need_b200(vec, "B200_lVector::ScaleAdd")),
          "B200_lVector::ScaleAdd");
}

// Plane rotation of (vec, this): vec' = c vec + s this, this' = c this - s vec
// (BLAS ?rot with x = vec, y = this, as GPUblas_lVector::Rot passes them).
template < typename T > void B200_lVector< T >::Rot(lVector< T > *vec, const T &sc, const T &ss) {
  B200_lVector< T > *o = dynamic_cast< B200_lVector< T > * >(vec);
  if (!o) fail("B200_lVector::Rot", "the other vector is not a B200 vector of the same value type");
  std::vector< T > x = o->download(), y = download();
  for (int i = 0; i < this->size_; ++i) {
    const T xi = x[i], yi = y[i];
    x[i] = sc * xi + ss * yi;
    y[i] = sc * yi - ss * xi;
  }
  o->upload(x);
  upload(y);
}

// Givens rotation (c, s) that zeroes b in (a, b): r = +-sqrt(a^2 + b^2) with
// the sign of the larger-magnitude input, c = a / r, s = b / r; a <- r and
// b <- z (the reconstruction scalar: s if |a| > |b|, 1/c if c != 0, else 1).
template < typename T > void B200_lVector< T >::Rotg(T *sa, T *sb, T *sc, T *ss) const {
  const T a = *sa, b = *sb;
  const T scale = std::abs(a) + std::abs(b);
  if (scale == T(0)) {
    *sc = T(1);
    *ss = T(0);
    *sa = T(0);
    *sb = T(0);
    return;
  }
  const T roe = std::abs(a) > std::abs(b) ? a : b;
  T r = scale * std::sqrt((a / scale) * (a / scale) + (b / scale) * (b / scale));
  if (roe < T(0)) r = -r;
  *sc = a / r;
  *ss = b / r;
  T z = T(1);
  if (std::abs(a) > std::abs(b)) z = *ss;
  else if (*sc != T(0)) z = T(1) / *sc;
  *sa = r;
  *sb = z;
}

template < typename T > void B200_lVector< T >::Rotm(lVector< T > *, const T &) {
  fail("B200_lVector::Rotm", "modified Givens rotations are not supported by the B200 backend");
}

template < typename T > void B200_lVector< T >::Rotmg(T *, T *, T *, const T &, T *) const {
  fail("B200_lVector::Rotmg", "modified Givens rotations are not supported by the B200 backend");
}

template < typename T > T *B200_lVector< T >::GetBuffer() const {
  if (!vec_) return nullptr;
  int64_t n = 0;
  int dt = 0;
  void *p = nullptr;
  check(b200la_vec_info(vec_, &n, &dt, &p), "B200_lVector::GetBuffer");
  return static_cast< T * >(p);
}

// ---------------------------------------------------------------- matrices

template < typename T > B200_CSR_lMatrix< T >::B200_CSR_lMatrix() {
  this->platform_name_ = "GPU (B200)";
  this->platform_id_ = GPU;
  this->implementation_name_ = "B200 (sm_100a)";
  this->implementation_id_ = B200;
  this->matrix_format_name_ = "CSR";
  this->matrix_format_id_ = CSR;
  this->num_row_ = this->num_col_ = this->nnz_ = 0;
  this->symmetric_ = false;
}

template < typename T > B200_CSR_lMatrix< T >::~B200_CSR_lMatrix() { this->Clear(); }

template < typename T >
void B200_CSR_lMatrix< T >::Init(const int init_nnz, const int init_num_row, const int init_num_col,
                                 const std::string init_name) {
  this->Clear();
  this->nnz_ = init_nnz;
  this->num_row_ = init_num_row;
  this->num_col_ = init_num_col;
  this->name_ = init_name;
}

template < typename T > void B200_CSR_lMatrix< T >::Clear(void) {
  if (mat_) b200la_mat_destroy(mat_);
  mat_ = nullptr;
  rowptr_.clear();
  col_.clear();
  this->nnz_ = this->num_row_ = this->num_col_ = 0;
}

template < typename T > void B200_CSR_lMatrix< T >::upload_values(const T *val) {
  if ((int)rowptr_.size() != this->num_row_ + 1)
    fail("B200_CSR_lMatrix::CopyFrom", "no structure: call CopyStructureFrom first");
  if (mat_) b200la_mat_destroy(mat_);
  mat_ = nullptr;
  check(b200la_csr_upload(b200_lmp_context(), this->num_row_, this->num_col_, this->nnz_, rowptr_.data(),
                          col_.data(), val, dtype_of< T >(), dtype_of< T >(), &mat_),
        "B200_CSR_lMatrix::CopyFrom");
}

template < typename T >
void B200_CSR_lMatrix< T >::download(std::vector< int > *rowptr, std::vector< int > *col, std::vector< T > *val) const {
  rowptr->resize(this->num_row_ + 1);
  col->resize(this->nnz_);
  val->resize(this->nnz_);
  if (!mat_) fail("B200_CSR_lMatrix", "the matrix holds no values");
  check(b200la_mat_download(mat_, rowptr->data(), col->data(), val->data()), "B200_CSR_lMatrix::CopyTo");
}

template < typename T > void B200_CSR_lMatrix< T >::Zeros(void) {
  std::vector< T > z(this->nnz_, T(0));
  upload_values(z.data());
}

template < typename T > void B200_CSR_lMatrix< T >::ZeroRows(const int *index_set, const int size, const T alpha) {
  if (!mat_) fail("B200_CSR_lMatrix::ZeroRows", "the matrix holds no values");
  check(b200la_mat_zero_rows(mat_, index_set, size, (double)alpha), "B200_CSR_lMatrix::ZeroRows");
}

template < typename T > lMatrix< T > &B200_CSR_lMatrix< T >::operator=(const lMatrix< T > &mat2) {
  if (this != &mat2) this->CopyFrom(mat2);
  return *this;
}

template < typename T > void B200_CSR_lMatrix< T >::CopyStructureFrom(const lMatrix< T > &mat2) {
  if (this == &mat2) return;
  this->Init(mat2.get_nnz(), mat2.get_num_row(), mat2.get_num_col(), mat2.get_name());
  if (const CPU_CSR_lMatrix< T > *c = dynamic_cast< const CPU_CSR_lMatrix< T > * >(&mat2)) {
    rowptr_.assign(c->matrix.row, c->matrix.row + this->num_row_ + 1);
    col_.assign(c->matrix.col, c->matrix.col + this->nnz_);
  } else if (const B200_CSR_lMatrix< T > *b = dynamic_cast< const B200_CSR_lMatrix< T > * >(&mat2)) {
    if (b->mat_) {
      std::vector< T > v;
      b->download(&rowptr_, &col_, &v);
    } else {
      rowptr_ = b->rowptr_;
      col_ = b->col_;
    }
  } else {
    mat2.CopyStructureTo(*this);
  }
}

template < typename T > void B200_CSR_lMatrix< T >::CopyStructureTo(lMatrix< T > &mat2) const {
  if (CPU_CSR_lMatrix< T > *c = dynamic_cast< CPU_CSR_lMatrix< T > * >(&mat2)) {
    // the CPU matrix takes its structure from a CPU copy of this one
    CPUsimple_CSR_lMatrix< T > tmp;
    tmp.Init(this->nnz_, this->num_row_, this->num_col_, this->name_);
    std::vector< int > rp, cl;
    std::vector< T > v;
    if (mat_) download(&rp, &cl, &v);
    else {
      rp = rowptr_;
      cl = col_;
    }
    std::copy(rp.begin(), rp.end(), tmp.matrix.row);
    std::copy(cl.begin(), cl.end(), tmp.matrix.col);
    c->CopyStructureFrom(tmp);
  } else {
    mat2.CopyStructureFrom(*this);
  }
}

template < typename T > void B200_CSR_lMatrix< T >::CopyFrom(const lMatrix< T > &mat2) {
  if (this == &mat2) return;
  assert(this->nnz_ == mat2.get_nnz() && this->num_row_ == mat2.get_num_row());
  if (const CPU_CSR_lMatrix< T > *c = dynamic_cast< const CPU_CSR_lMatrix< T > * >(&mat2)) {
    upload_values(c->matrix.val);
  } else if (const B200_CSR_lMatrix< T > *b = dynamic_cast< const B200_CSR_lMatrix< T > * >(&mat2)) {
    std::vector< int > rp, cl;
    std::vector< T > v;
    b->download(&rp, &cl, &v);
    rowptr_ = rp;
    col_ = cl;
    upload_values(v.data());
  } else {
    mat2.CopyTo(*this);
  }
}

template < typename T > void B200_CSR_lMatrix< T >::CopyTo(lMatrix< T > &mat2) const {
  if (CPU_CSR_lMatrix< T > *c = dynamic_cast< CPU_CSR_lMatrix< T > * >(&mat2)) {
    assert(this->nnz_ == mat2.get_nnz() && this->num_row_ == mat2.get_num_row());
    std::vector< int > rp, cl;
    std::vector< T > v;
    download(&rp, &cl, &v);
    std::copy(v.begin(), v.end(), c->matrix.val);
  } else {
    mat2.CopyFrom(*this);
  }
}

namespace {
template < typename T, typename S > void mat_cast_into(B200_CSR_lMatrix< T > &dst, const lMatrix< S > &src) {
  if (const B200_CSR_lMatrix< S > *b = dynamic_cast< const B200_CSR_lMatrix< S > * >(&src)) {
    // the same structure, values converted on the device (CastFrom)
    b200la_mat m = nullptr;
    if (!b->handle()) fail("B200_CSR_lMatrix::CastFrom", "the source holds no values");
    check(b200la_mat_cast(b->handle(), dtype_of< T >(), &m), "B200_CSR_lMatrix::CastFrom");
    std::vector< int > rp(src.get_num_row() + 1), cl(src.get_nnz());
    std::vector< T > v(src.get_nnz());
    check(b200la_mat_download(m, rp.data(), cl.data(), v.data()), "B200_CSR_lMatrix::CastFrom");
    b200la_mat_destroy(m);
    CPUsimple_CSR_lMatrix< T > tmp;
    tmp.Init(src.get_nnz(), src.get_num_row(), src.get_num_col(), src.get_name());
    std::copy(rp.begin(), rp.end(), tmp.matrix.row);
    std::copy(cl.begin(), cl.end(), tmp.matrix.col);
    std::copy(v.begin(), v.end(), tmp.matrix.val);
    dst.CopyStructureFrom(tmp);
    dst.CopyFrom(tmp);
  } else if (const CPU_CSR_lMatrix< S > *c = dynamic_cast< const CPU_CSR_lMatrix< S > * >(&src)) {
    CPUsimple_CSR_lMatrix< T > tmp;
    tmp.Init(src.get_nnz(), src.get_num_row(), src.get_num_col(), src.get_name());
    std::copy(c->matrix.row, c->matrix.row + src.get_num_row() + 1, tmp.matrix.row);
    std::copy(c->matrix.col, c->matrix.col + src.get_nnz(), tmp.matrix.col);
    for (int k = 0; k < src.get_nnz(); ++k) tmp.matrix.val[k] = (T)c->matrix.val[k];
    dst.CopyStructureFrom(tmp);
    dst.CopyFrom(tmp);
  } else {
    src.CastTo(dst);
  }
}
} // namespace

template < typename T > void B200_CSR_lMatrix< T >::CastFrom(const lMatrix< double > &other) {
  mat_cast_into(*this, other);
}
template < typename T > void B200_CSR_lMatrix< T >::CastFrom(const lMatrix< float > &other) {
  mat_cast_into(*this, other);
}

template < typename T > void B200_CSR_lMatrix< T >::CastTo(lMatrix< double > &other) const { other.CastFrom(*this); }
template < typename T > void B200_CSR_lMatrix< T >::CastTo(lMatrix< float > &other) const { other.CastFrom(*this); }

template < typename T > void B200_CSR_lMatrix< T >::ConvertFrom(const lMatrix< T > &mat2) {
  // CSR from a CPU COO matrix: TransformFromCOO on the device, the
  // reference's CSR bit for bit (b200la_coo_upload)
  if (const CPU_COO_lMatrix< T > *c = dynamic_cast< const CPU_COO_lMatrix< T > * >(&mat2)) {
    this->Init(c->get_nnz(), c->get_num_row(), c->get_num_col(), c->get_name());
    if (mat_) b200la_mat_destroy(mat_);
    mat_ = nullptr;
    check(b200la_coo_upload(b200_lmp_context(), this->num_row_, this->num_col_, this->nnz_, c->matrix.row,
                            c->matrix.col, c->matrix.val, dtype_of< T >(), dtype_of< T >(), 0, &mat_),
          "B200_CSR_lMatrix::ConvertFrom");
    std::vector< T > v;
    download(&rowptr_, &col_, &v);
  } else {
    fail("B200_CSR_lMatrix::ConvertFrom", "unsupported matrix type (a CPU COO matrix is expected)");
  }
}

template < typename T > lMatrix< T > *B200_CSR_lMatrix< T >::CloneWithoutContent(void) const {
  B200_CSR_lMatrix< T > *m = new B200_CSR_lMatrix< T >();
  m->Init(this->nnz_, this->num_row_, this->num_col_, "clone from " + this->name_);
  return m;
}

template < typename T > void B200_CSR_lMatrix< T >::Sync(void) const {
  check(b200la_ctx_synchronize(b200_lmp_context()), "B200_CSR_lMatrix::Sync");
}

template < typename T > void B200_CSR_lMatrix< T >::Tune() {
  if (!mat_) fail("B200_CSR_lMatrix::Tune", "the matrix holds no values");
  check(b200la_mat_tune(mat_, nullptr, nullptr, nullptr), "B200_CSR_lMatrix::Tune");
}

template < typename T >
void B200_CSR_lMatrix< T >::VectorMult(const lVector< T > &invec, lVector< T > *outvec) const {
  if (!mat_) fail("B200_CSR_lMatrix::VectorMult", "the matrix holds no values");
  check(b200la_spmv(mat_, need_b200(invec, "B200_CSR_lMatrix::VectorMult"),
                    need_b200(*outvec, "B200_CSR_lMatrix::VectorMult")),
        "B200_CSR_lMatrix::VectorMult");
}

template < typename T >
void B200_CSR_lMatrix< T >::VectorMultAdd(const lVector< T > &invec, lVector< T > *outvec) const {
  if (!mat_) fail("B200_CSR_lMatrix::VectorMultAdd", "the matrix holds no values");
  check(b200la_spmv_add(mat_, need_b200(invec, "B200_CSR_lMatrix::VectorMultAdd"),
                        need_b200(*outvec, "B200_CSR_lMatrix::VectorMultAdd")),
        "B200_CSR_lMatrix::VectorMultAdd");
}

template < typename T >
void B200_CSR_lMatrix< T >::VectorMultNoDiag(const lVector< T > &in, lVector< T > *out) const {
  if (!mat_) fail("B200_CSR_lMatrix::VectorMultNoDiag", "the matrix holds no values");
  check(b200la_spmv_nodiag(mat_, need_b200(in, "B200_CSR_lMatrix::VectorMultNoDiag"),
                           need_b200(*out, "B200_CSR_lMatrix::VectorMultNoDiag")),
        "B200_CSR_lMatrix::VectorMultNoDiag");
}

template < typename T >
void B200_CSR_lMatrix< T >::extract_invdiagelements(const int start_i, const int end_i, lVector< T > *vec) const {
  if (!mat_) fail("B200_CSR_lMatrix::extract_invdiagelements", "the matrix holds no values");
  if (start_i == 0 && end_i == this->num_row_) {
    if (B200_lVector< T > *b = dynamic_cast< B200_lVector< T > * >(vec)) {
      check(b200la_mat_inv_diag(mat_, b->handle()), "B200_CSR_lMatrix::extract_invdiagelements");
      return;
    }
  }
  // a row range or a non-B200 target: through a device vector of all rows
  B200_lVector< T > all(this->num_row_, "inverse diagonal");
  check(b200la_mat_inv_diag(mat_, all.handle()), "B200_CSR_lMatrix::extract_invdiagelements");
  std::vector< T > h(end_i - start_i);
  all.GetBlockValues(start_i, end_i, h.data());
  std::vector< int > idx(end_i - start_i);
  for (int k = 0; k < end_i - start_i; ++k) idx[k] = k;
  vec->SetValues(idx.data(), (int)idx.size(), h.data());
}

template < typename T > void B200_CSR_lMatrix< T >::SwapDiagElementsToRowFront(void) {
  // CPU_CSR_lMatrix::SwapDiagElementsToRowFront: the diagonal entry of each
  // row moves to the row's first position (swapped with the entry there)
  std::vector< int > rp, cl;
  std::vector< T > v;
  download(&rp, &cl, &v);
  for (int i = 0; i < this->num_row_; ++i)
    for (int j = rp[i]; j < rp[i + 1]; ++j)
      if (cl[j] == i) {
        std::swap(cl[j], cl[rp[i]]);
        std::swap(v[j], v[rp[i]]);
        break;
      }
  rowptr_ = rp;
  col_ = cl;
  upload_values(v.data());
}

// ---------------------------------------------------------------- factories

template < typename T >
lVector< T > *init_vector_b200(const int size, const std::string name, const enum PLATFORM &platform,
                               const enum IMPLEMENTATION &implementation) {
  if (implementation == B200) return new B200_lVector< T >(size, name);
  return init_vector< T >(size, name, platform, implementation);
}

template < typename T >
lMatrix< T > *init_matrix_b200(const int init_nnz, const int init_num_row, const int init_num_col,
                               const std::string init_name, const enum PLATFORM &platform,
                               const enum IMPLEMENTATION &implementation, const enum MATRIX_FORMAT &matrix_format) {
  if (implementation == B200) {
    if (matrix_format != CSR) fail("init_matrix_b200", "the B200 backend stores CSR matrices");
    B200_CSR_lMatrix< T > *m = new B200_CSR_lMatrix< T >();
    m->Init(init_nnz, init_num_row, init_num_col, init_name);
    return m;
  }
  return init_matrix< T >(init_nnz, init_num_row, init_num_col, init_name, platform, implementation, matrix_format);
}

template class B200_lVector< double >;
template class B200_lVector< float >;
template class B200_CSR_lMatrix< double >;
template class B200_CSR_lMatrix< float >;
template lVector< double > *init_vector_b200< double >(const int, const std::string, const enum PLATFORM &,
                                                       const enum IMPLEMENTATION &);
template lVector< float > *init_vector_b200< float >(const int, const std::string, const enum PLATFORM &,
                                                     const enum IMPLEMENTATION &);
template lMatrix< double > *init_matrix_b200< double >(const int, const int, const int, const std::string,
                                                       const enum PLATFORM &, const enum IMPLEMENTATION &,
                                                       const enum MATRIX_FORMAT &);
template lMatrix< float > *init_matrix_b200< float >(const int, const int, const int, const std::string,
                                                     const enum PLATFORM &, const enum IMPLEMENTATION &,
                                                     const enum MATRIX_FORMAT &);

} // namespace la
} // namespace hiflow
