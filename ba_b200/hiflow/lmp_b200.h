// HiFlow3 lmp backend on B200: B200_lVector<T> and B200_CSR_lMatrix<T>
// implement HiFlow3's lVector<T> (linear_algebra/lmp/lvector.h:38-321) and
// CSR_lMatrix<T> (lmp/lmatrix_csr.h:27, lmp/lmatrix.h:39-468) over the
// b200la C ABI (include/b200la.h), so that lmp code written against those
// interfaces -- the lmp cg() (lmp/solvers/cg.h:93-209), lPreconditioner_Jacobi
// (lmp/lpreconditioner.cc:125-200), the CoupledVector/CoupledMatrix blocks --
// runs on the GPU unchanged.  This file is compiled inside HiFlow3's own
// source tree (it includes HiFlow3's lmp headers); it does not depend on
// anything else of this repository but the b200la library.
//
// Platform and implementation: PLATFORM GPU with a new IMPLEMENTATION value
// B200 (la_global.h:43-54 ends at PETSC; B200 is the next value).  The
// factories init_vector_b200 / init_matrix_b200 return the B200 classes for
// IMPLEMENTATION B200 and defer to HiFlow3's init_vector / init_matrix
// (lmp/init_vec_mat.cc:146,259) for everything else; HiFlow3 adds the same two
// cases to those factories to make B200 selectable from its parameters.
//
// Device context: one b200la context per process, on the device set by
// b200_lmp_set_device (default 0), created at the first B200 object.
//
// Memory and copies follow the GPU_lVector / GPU_CSR_lMatrix conventions
// (lmp/cuda/lvector_gpu.cc, lmatrix_csr_gpu.cc): Init allocates device memory,
// CopyFrom / CopyTo move data between a CPU object and a B200 object
// (dynamic_cast on the other side, as CPU_CSR_lMatrix::CopyFrom does,
// lmp/lmatrix_csr_cpu.cc:210-240), CopyStructureFrom takes the sparsity
// pattern of a CPU CSR matrix.  Errors follow the reference: LOG_ERROR with
// the b200la message, then quit_program() (lmp/cuda/cuda_utils.h:24-55 exits
// the same way).
#ifndef HIFLOW_LINEAR_ALGEBRA_LMP_LMP_B200_H
#define HIFLOW_LINEAR_ALGEBRA_LMP_LMP_B200_H

#include <string>
#include <vector>

#include "b200la.h"
#include "init_vec_mat.h"
#include "lmatrix_csr.h"
#include "lvector.h"

namespace hiflow {
namespace la {

/// IMPLEMENTATION value of the B200 backend (the next value after PETSC).
constexpr IMPLEMENTATION B200 = static_cast< IMPLEMENTATION >(PETSC + 1);

/// Device of the process-wide b200la context (call before the first B200
/// object is created).
void b200_lmp_set_device(int device);
/// The process-wide b200la context (created on first use).
b200la_ctx b200_lmp_context();

template < typename ValueType > class B200_lVector : public lVector< ValueType > {
public:
  B200_lVector();
  B200_lVector(int size, const std::string &name);
  virtual ~B200_lVector();

  // element access (host round trips; not on the solver path)
  virtual void add_value(const int i, ValueType val);
  virtual void add_values(const int *indices, int length, const ValueType *values);
  virtual void SetValues(const int *index, const int size, const ValueType *values);
  virtual void SetValue(const int index, const ValueType value);
  virtual void GetValues(const int *index, const int size, ValueType *values) const;
  virtual ValueType GetValue(const int index) const;
  virtual void SetBlockValues(const int start_i, const int end_i, const ValueType *values);
  virtual void GetBlockValues(const int start_i, const int end_i, ValueType *values) const;
  virtual void set_indexset(const int *indexset, const int size);
  virtual void get_indexset(int *indexset) const;
  virtual int get_indexset_size(void) const;
  virtual void GetIndexedValues(ValueType *values) const;
  virtual void SetIndexedValues(const ValueType *values);
  virtual lVector< ValueType > *extract_subvector(const int start_i, const int end_i) const;
  virtual void partial_replace_subvector(const int start_i, const int start_sub_vec, const int size,
                                         const lVector< ValueType > &sub_vec);
  virtual void partial_add_subvector(const int start_i, const int start_sub_vec, const int size,
                                     const ValueType weight, const lVector< ValueType > &sub_vec);

  virtual void Init(const int size, const std::string name);
  virtual void Clear(void);
  virtual void Zeros(void);
  virtual void Reorder(const int *index);

  virtual lVector< ValueType > &operator=(const lVector< ValueType > &vec2);
  virtual void CopyFrom(const lVector< ValueType > &vec);
  virtual void CopyTo(lVector< ValueType > &vec) const;
  virtual void CastFrom(const lVector< double > &vec);
  virtual void CastFrom(const lVector< float > &vec);
  virtual void CastTo(lVector< double > &vec) const;
  virtual void CastTo(lVector< float > &vec) const;
  virtual lVector< ValueType > *CloneWithoutContent(void) const;
  virtual void Sync(void) const;

  // BLAS-1 on the device
  virtual void ElementWiseMult(const lVector< ValueType > &vec) const;
  virtual int ArgMin(void) const;
  virtual int ArgMax(void) const;
  virtual ValueType Norm1(void) const;
  virtual ValueType Norm2(void) const;
  virtual ValueType NormMax(void) const;
  virtual ValueType Dot(const lVector< ValueType > &vec) const;
  virtual void Scale(const ValueType scalar);
  virtual void Axpy(const lVector< ValueType > &vec, const ValueType scalar);
  virtual void ScaleAdd(const ValueType scalar, const lVector< ValueType > &vec);
  virtual void Rot(lVector< ValueType > *vec, const ValueType &sc, const ValueType &ss);
  virtual void Rotg(ValueType *sa, ValueType *sb, ValueType *sc, ValueType *ss) const;
  virtual void Rotm(lVector< ValueType > *vec, const ValueType &sparam);
  virtual void Rotmg(ValueType *sd1, ValueType *sd2, ValueType *x1, const ValueType &x2,
                     ValueType *sparam) const;
  /// The device buffer (as GPU_lVector::buffer, lmp/cuda/lvector_gpu.h:118).
  virtual ValueType *GetBuffer() const;
  virtual bool ContainsNaN() const;

  /// The b200la vector handle (for b200la calls on this vector).
  b200la_vec handle() const { return vec_; }

private:
  std::vector< ValueType > download() const;
  void upload(const std::vector< ValueType > &h);
  b200la_vec vec_ = nullptr;
  std::vector< int > indexset_;
};

template < typename ValueType > class B200_CSR_lMatrix : public CSR_lMatrix< ValueType > {
public:
  B200_CSR_lMatrix();
  virtual ~B200_CSR_lMatrix();

  virtual void Init(const int init_nnz, const int init_num_row, const int init_num_col,
                    const std::string init_name);
  virtual void Clear(void);
  virtual void Zeros(void);
  virtual void ZeroRows(const int *index_set, const int size, const ValueType alpha);

  virtual lMatrix< ValueType > &operator=(const lMatrix< ValueType > &mat2);
  virtual void CopyFrom(const lMatrix< ValueType > &mat2);
  virtual void CopyTo(lMatrix< ValueType > &mat2) const;
  virtual void CastFrom(const lMatrix< double > &other);
  virtual void CastFrom(const lMatrix< float > &other);
  virtual void CastTo(lMatrix< double > &other) const;
  virtual void CastTo(lMatrix< float > &other) const;
  virtual void ConvertFrom(const lMatrix< ValueType > &mat2);
  virtual void CopyStructureFrom(const lMatrix< ValueType > &mat2);
  virtual void CopyStructureTo(lMatrix< ValueType > &mat2) const;
  virtual lMatrix< ValueType > *CloneWithoutContent(void) const;
  virtual void Sync(void) const;

  virtual void VectorMult(const lVector< ValueType > &invec, lVector< ValueType > *outvec) const;
  virtual void VectorMultAdd(const lVector< ValueType > &invec, lVector< ValueType > *outvec) const;
  virtual void VectorMultNoDiag(const lVector< ValueType > &in, lVector< ValueType > *out) const;
  virtual void extract_invdiagelements(const int start_i, const int end_i, lVector< ValueType > *vec) const;
  virtual void SwapDiagElementsToRowFront(void);

  /// Schedule of the device SpMV: b200la_mat_tune's pick (format, parameter).
  void Tune();
  /// The b200la matrix handle (nullptr until values were copied in).
  b200la_mat handle() const { return mat_; }

private:
  void upload_values(const ValueType *val);
  void download(std::vector< int > *rowptr, std::vector< int > *col, std::vector< ValueType > *val) const;
  b200la_mat mat_ = nullptr;
  // the sparsity pattern from CopyStructureFrom, held until the values come
  std::vector< int > rowptr_, col_;
};

/// init_vector / init_matrix (lmp/init_vec_mat.cc:146,259) with the B200
/// cases: IMPLEMENTATION B200 (with PLATFORM GPU, format CSR) gives the B200
/// classes, any other combination goes to HiFlow3's factories.
template < typename ValueType >
lVector< ValueType > *init_vector_b200(const int size, const std::string name, const enum PLATFORM &platform,
                                       const enum IMPLEMENTATION &implementation);
template < typename ValueType >
lMatrix< ValueType > *init_matrix_b200(const int init_nnz, const int init_num_row, const int init_num_col,
                                       const std::string init_name, const enum PLATFORM &platform,
                                       const enum IMPLEMENTATION &implementation,
                                       const enum MATRIX_FORMAT &matrix_format);

} // namespace la
} // namespace hiflow

#endif
