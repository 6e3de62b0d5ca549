// Drop-in LinAlg::Dense<Scalar> (the reference's include/LinAlg/dense.hpp:46-133):
// column-major host matrix, element (i, j) at data[i + j*m] (src/LinAlg/dense.cpp:298).
#pragma once
#ifndef MFGPU_LINALG_DENSE_HPP
#define MFGPU_LINALG_DENSE_HPP 1

#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <utility>
#include <vector>

#include "vec.hpp"

namespace LinAlg {

template <class Scalar>
class Dense {
 public:
  Dense(int m = 0, int n = 0) : m_(0), n_(0) { resize(m, n); }
  Dense(const Dense& A) = default;
  // Submatrix A(rows, cols) (dense.cpp:67-86).
  Dense(const Dense& A, const IdxVec& rows, const IdxVec& cols)
      : m_((int)rows.size()), n_((int)cols.size()), data_(rows.size() * cols.size()) {
    for (int j = 0; j < n_; j++)
      for (int i = 0; i < m_; i++) (*this)(i, j) = A(rows[i], cols[j]);
  }
  void resize(int m, int n) {
    if (m < 0 || n < 0) throw std::domain_error("Matrix dimensions must be positive!");
    m_ = m;
    n_ = n;
    data_.resize((size_t)m * n);
  }
  Dense& operator=(Dense A) {
    swap(A);
    return *this;
  }
  Dense& operator+=(const Dense& A) {
    check(A);
    for (size_t i = 0; i < data_.size(); i++) data_[i] += A.data_[i];
    return *this;
  }
  Dense& operator-=(const Dense& A) {
    check(A);
    for (size_t i = 0; i < data_.size(); i++) data_[i] -= A.data_[i];
    return *this;
  }
  Dense& operator*=(const Scalar& a) {
    for (Scalar& x : data_) x *= a;
    return *this;
  }
  Dense& operator/=(const Scalar& a) {
    const Scalar ai = Scalar(1) / a;
    for (Scalar& x : data_) x *= ai;
    return *this;
  }
  // C = A * B (dgemm in the reference, dense.cpp:151-163)
  Dense operator*(const Dense& B) const {
    if (n_ != B.m_) throw std::invalid_argument("Dense: inner dimensions differ");
    Dense C(m_, B.n_);
    for (int j = 0; j < B.n_; j++)
      for (int k = 0; k < n_; k++) {
        const Scalar b = B(k, j);
        if (b == Scalar(0)) continue;
        for (int i = 0; i < m_; i++) C(i, j) += (*this)(i, k) * b;
      }
    return C;
  }
  // y = A * v (dgemv, dense.cpp:208-218)
  Vec<Scalar> operator*(const Vec<Scalar>& v) const {
    if (n_ != v.n()) throw std::invalid_argument("Dense: vector length differs");
    Vec<Scalar> y(m_);
    for (int j = 0; j < n_; j++)
      for (int i = 0; i < m_; i++) y(i) += (*this)(i, j) * v(j);
    return y;
  }
  double norm() const {   // Frobenius norm (dnrm2 over the storage)
    Vec<Scalar> v((int)data_.size());
    for (size_t i = 0; i < data_.size(); i++) v((int)i) = data_[i];
    return v.norm();
  }
  Scalar& operator()(int i, int j) { return data_[i + (size_t)j * m_]; }
  const Scalar& operator()(int i, int j) const { return data_[i + (size_t)j * m_]; }
  Dense operator()(const IdxVec& rows, const IdxVec& cols) { return Dense(*this, rows, cols); }
  void print() const {
    std::cout << m_ << " " << n_ << std::endl;
    for (int i = 0; i < m_; i++) {
      for (int j = 0; j < n_; j++)
        std::cout << " " << std::fixed << std::setprecision(4) << std::setw(8) << (*this)(i, j);
      std::cout << std::endl;
    }
  }
  int m() const { return m_; }
  int n() const { return n_; }
  void swap(Dense& o) {
    std::swap(m_, o.m_);
    std::swap(n_, o.n_);
    std::swap(data_, o.data_);
  }
  Scalar* data() { return data_.data(); }
  const Scalar* data() const { return data_.data(); }

 private:
  void check(const Dense& A) const {
    if (A.m_ != m_ || A.n_ != n_) throw std::invalid_argument("Dense: size mismatch");
  }
  int m_, n_;
  std::vector<Scalar> data_;
};

}  // namespace LinAlg
#endif
