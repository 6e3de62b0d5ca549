// Drop-in LinAlg::Sparse<Scalar> (the reference's include/LinAlg/sparse.hpp:33-83):
// CSR storage with the same constructor, accessors, dense sub-block extraction
// and matrix-vector product.
#pragma once
#ifndef MFGPU_LINALG_SPARSE_HPP
#define MFGPU_LINALG_SPARSE_HPP 1

#include <iostream>
#include <stdexcept>
#include <vector>

#include "dense.hpp"
#include "vec.hpp"

namespace LinAlg {

template <class Scalar>
class Sparse {
 public:
  Sparse() : m_(0), n_(0), nnz_(0) {}
  // Sparse(val, col_ind, row_ptr, m, n) (sparse.cpp:46-55): nnz = row_ptr[m].
  Sparse(const std::vector<Scalar>& val, const IdxVec& col_ind, const IdxVec& row_ptr, int m, int n)
      : m_(m), n_(n), val_(val), col_ind_(col_ind), row_ptr_(row_ptr) {
    if ((int)row_ptr_.size() != m_ + 1) throw std::invalid_argument("Sparse: row_ptr size != m+1");
    nnz_ = row_ptr_[m_];
  }
  Sparse(const Sparse& o) = default;
  void operator=(Sparse o) {
    m_ = o.m_;
    n_ = o.n_;
    nnz_ = o.nnz_;
    val_.swap(o.val_);
    col_ind_.swap(o.col_ind_);
    row_ptr_.swap(o.row_ptr_);
  }
  // y = A v (sparse.cpp:62-77), row sums in CSR order
  Vec<Scalar> operator*(const Vec<Scalar>& v) const {
    Vec<Scalar> y(m_);
    for (int i = 0; i < m_; i++) {
      Scalar s = 0;
      for (int p = row_ptr_[i]; p < row_ptr_[i + 1]; p++) s += val_[p] * v(col_ind_[p]);
      y(i) = s;
    }
    return y;
  }
  const Scalar operator()(int i, int j) const {
    for (int p = row_ptr_[i]; p < row_ptr_[i + 1]; p++)
      if (col_ind_[p] == j) return val_[p];
    return 0;
  }
  int m() const { return m_; }
  int n() const { return n_; }
  int nnz() const { return nnz_; }
  Scalar val(int i) const { return val_[i]; }
  int col_ind(int i) const { return col_ind_[i]; }
  int row_ptr(int i) const { return row_ptr_[i]; }
  // dense sub-block A(rows, cols) (sparse.cpp:95-116)
  Dense<Scalar> operator()(const IdxVec& rows, const IdxVec& cols) const {
    Dense<Scalar> B((int)rows.size(), (int)cols.size());
    for (size_t ii = 0; ii < rows.size(); ii++)
      for (size_t jj = 0; jj < cols.size(); jj++) B((int)ii, (int)jj) = (*this)(rows[ii], cols[jj]);
    return B;
  }
  double norm() const {
    Vec<Scalar> v((int)val_.size());
    for (size_t i = 0; i < val_.size(); i++) v((int)i) = val_[i];
    return v.norm();
  }
  void print() const {
    std::cout << m_ << " " << n_ << std::endl;
    for (int i = 0; i < m_; i++)
      for (int p = row_ptr_[i]; p < row_ptr_[i + 1]; p++)
        std::cout << "(i,j,a) = (" << i << "," << col_ind_[p] << "," << val_[p] << ")" << std::endl;
  }
  // raw CSR (not in the reference): for the C ABI
  const Scalar* valData() const { return val_.data(); }
  const int* colIndData() const { return col_ind_.data(); }
  const int* rowPtrData() const { return row_ptr_.data(); }

 private:
  int m_, n_, nnz_;
  std::vector<Scalar> val_;
  IdxVec col_ind_;
  IdxVec row_ptr_;
};

}  // namespace LinAlg
#endif
