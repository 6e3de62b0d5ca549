// Drop-in LinAlg::Vec<Scalar> (the reference's include/LinAlg/vec.hpp:34-90):
// a host vector with the same constructors, operators and utility indexing.
// Arithmetic is plain host code; the factorization work runs on the GPU
// behind TreeFactor2D::MF2D / TreeFactor3D::MF3D (DE/mf.hpp).
#pragma once
#ifndef MFGPU_LINALG_VEC_HPP
#define MFGPU_LINALG_VEC_HPP 1

// The reference's LinAlg headers pull these in; callers (including its own
// fixtures, which use assert) rely on them transitively.
#include <assert.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <utility>
#include <vector>

typedef std::vector<int> IdxVec;
typedef std::complex<double> dcomplex;

namespace LinAlg {
template <typename U> class Dense;
template <typename U> class Sparse;

template <class Scalar>
class Vec {
 public:
  friend class Dense<Scalar>;
  friend class Sparse<Scalar>;
  // Vec(int n = 0) (vec.hpp:45): n zeros; negative sizes throw std::domain_error.
  Vec(int n = 0) : n_(0) { resize(n); }
  Vec(const Vec& v) : n_(v.n_), data_(v.data_) {}
  // Subvector v(idxs) (vec.hpp:51, src/LinAlg/vec.cpp:41-52).
  Vec(const Vec& v, const IdxVec& idxs) : n_((int)idxs.size()), data_(idxs.size()) {
    for (size_t i = 0; i < idxs.size(); i++) data_[i] = v.data_[idxs[i]];
  }
  Vec& operator=(Vec v) {
    swap(v);
    return *this;
  }
  Vec& operator+=(const Vec& v) {
    check(v);
    for (int i = 0; i < n_; i++) data_[i] += v.data_[i];
    return *this;
  }
  Vec& operator-=(const Vec& v) {
    check(v);
    for (int i = 0; i < n_; i++) data_[i] -= v.data_[i];
    return *this;
  }
  Vec& operator*=(const Scalar& a) {
    for (Scalar& x : data_) x *= a;
    return *this;
  }
  Vec& operator/=(const Scalar& a) {
    const Scalar ai = Scalar(1) / a;   // the reference scales by the reciprocal (vec.cpp:117-122)
    for (Scalar& x : data_) x *= ai;
    return *this;
  }
  // Euclidean norm (dnrm2 in the reference, vec.cpp:134-138), overflow-safe.
  double norm() const {
    double scale = 0.0, ssq = 1.0;
    for (const Scalar& x : data_) {
      const double a = std::abs(x);
      if (a == 0.0) continue;
      if (scale < a) {
        ssq = 1.0 + ssq * (scale / a) * (scale / a);
        scale = a;
      } else {
        ssq += (a / scale) * (a / scale);
      }
    }
    return scale * std::sqrt(ssq);
  }
  void resize(int n) {
    if (n < 0) throw std::domain_error("Matrix dimensions must be positive!");
    if (n > 0) {
      data_.resize(n);
      n_ = n;
    }
  }
  // b.set(idxs, vals): scatter (vec.cpp:4-12)
  void set(const IdxVec& idxs, const Vec& vals) {
    for (size_t i = 0; i < idxs.size(); i++) data_[idxs[i]] = vals.data_[i];
  }
  Scalar& operator()(int i) { return data_[i]; }
  const Scalar& operator()(int i) const { return data_[i]; }
  Vec operator()(const IdxVec& idxs) { return Vec(*this, idxs); }
  void print() const {
    std::cout << n_ << std::endl;
    for (int i = 0; i < n_; i++) {
      Scalar v = data_[i];
      if (std::abs(v) <= 1e-8) v = 0;
      std::cout << " " << v;
    }
    std::cout << std::endl;
  }
  void swap(Vec& o) {
    std::swap(n_, o.n_);
    std::swap(data_, o.data_);
  }
  int n() const { return n_; }
  // Contiguous storage (not in the reference): lets callers hand the vector
  // to the C ABI without a copy.
  Scalar* data() { return data_.data(); }
  const Scalar* data() const { return data_.data(); }

 private:
  void check(const Vec& v) const {
    if (v.n_ != n_) throw std::invalid_argument("Vec: size mismatch");
  }
  int n_;
  std::vector<Scalar> data_;
};

}  // namespace LinAlg
#endif
