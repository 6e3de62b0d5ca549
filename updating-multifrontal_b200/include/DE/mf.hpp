// Drop-in TreeFactor2D::MF2D<double> / TreeFactor3D::MF3D<double> (the
// reference's include/DE/mf.hpp:67-80 and 173-188): same constructors and
// public members (Factor, Update, Solve, Apply) and the same exception types,
// backed by the B200 implementation behind the C ABI of mfgpu.h.  The
// factorization lives in GPU memory owned by the object; Solve / Apply copy
// the vector in and out.  Only Scalar = double is provided.
//
// Build: -I<repo>/updating-multifrontal_b200/include/LinAlg
//        -I<repo>/updating-multifrontal_b200/include/DE -I<repo>/include
//        -L<repo>/updating-multifrontal_b200/lib -lmfgpu
// Environment: MFGPU_PRECISION=mixed selects the mixed-precision factorization
// with FP64 refinement; MFGPU_DEVICE=<n> the CUDA device.
#ifndef MFGPU_TREEFACTOR_MF_HPP
#define MFGPU_TREEFACTOR_MF_HPP 1

#include <cstdlib>
#include <set>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "linalg.hpp"
#include "mfgpu.h"

#ifndef LINE
#define LINE "--------------------------------------------------------------------------------"
#endif

namespace mfgpu_dropin {

// Status -> the reference's exception types: a too-shallow tree or broken
// leaf arithmetic is std::runtime_error (src/DE/mf2d.cpp:42,64); bad arguments
// std::invalid_argument; device failures and non-SPD input std::runtime_error.
inline void raise(int st, const char* msg) {
  if (st == MFGPU_OK) return;
  if (st == MFGPU_ERR_DEPTH || st == MFGPU_ERR_LEAF) throw std::runtime_error(msg);
  if (st == MFGPU_ERR_ARG) throw std::invalid_argument(msg);
  throw std::runtime_error(std::string(mfgpu_status_string(st)) + ": " + msg);
}

template <class Scalar>
class MFBase {
  static_assert(std::is_same<Scalar, double>::value,
                "the GPU multifrontal path computes in double precision (Scalar = double)");

 public:
  MFBase(const MFBase&) = delete;
  MFBase& operator=(const MFBase&) = delete;
  ~MFBase() { mfgpu_destroy(h_); }

  void Factor() { check(mfgpu_factor(h_)); }

  void Update(const LinAlg::Sparse<Scalar>& A, std::set<int> modifiedDOFs) {
    std::vector<int> mod(modifiedDOFs.begin(), modifiedDOFs.end());
    check(mfgpu_update(h_, A.valData(), A.nnz(), mod.data(), (int)mod.size()));
  }

  LinAlg::Vec<Scalar> Solve(const LinAlg::Vec<Scalar>& b) {
    LinAlg::Vec<Scalar> x(b.n());
    check(mfgpu_solve(h_, b.data(), x.data(), 1, b.n()));
    return x;
  }

  LinAlg::Vec<Scalar> Apply(const LinAlg::Vec<Scalar>& x) {
    LinAlg::Vec<Scalar> b(x.n());
    check(mfgpu_apply(h_, x.data(), b.data(), 1, x.n()));
    return b;
  }

  // The C ABI handle, for device-pointer solves, streams and statistics.
  mfgpu_handle* handle() { return h_; }

 protected:
  MFBase(int dim, const LinAlg::Sparse<Scalar>& A, int Nx, int Ny, int Nz, int width,
         int maxSideLength) {
    mfgpu_options o;
    mfgpu_default_options(&o);
    if (const char* p = std::getenv("MFGPU_PRECISION"))
      o.precision = std::string(p) == "mixed" ? MFGPU_MIXED : MFGPU_FP64;
    if (const char* d = std::getenv("MFGPU_DEVICE")) o.device = std::atoi(d);
    int st = mfgpu_create(dim, Nx, Ny, Nz, width, maxSideLength, A.m(), A.rowPtrData(),
                          A.colIndData(), A.valData(), &o, &h_);
    if (st != MFGPU_OK) raise(st, mfgpu_last_error(nullptr));
  }

 private:
  void check(int st) {
    if (st != MFGPU_OK) raise(st, mfgpu_last_error(h_));
  }
  mfgpu_handle* h_ = nullptr;
};

}  // namespace mfgpu_dropin

namespace TreeFactor2D {
// MF2D(A, Nx, Ny, width, maxSideLength) — include/DE/mf.hpp:74
template <class Scalar>
class MF2D : public mfgpu_dropin::MFBase<Scalar> {
 public:
  MF2D(const LinAlg::Sparse<Scalar>& A, int Nx, int Ny, int width = 1, int maxSideLength = 4)
      : mfgpu_dropin::MFBase<Scalar>(2, A, Nx, Ny, 1, width, maxSideLength) {}
};
}  // namespace TreeFactor2D

namespace TreeFactor3D {
// MF3D(A, Nx, Ny, Nz, width, maxSideLength) — include/DE/mf.hpp:180
template <class Scalar>
class MF3D : public mfgpu_dropin::MFBase<Scalar> {
 public:
  MF3D(const LinAlg::Sparse<Scalar>& A, int Nx, int Ny, int Nz, int width = 1,
       int maxSideLength = 4)
      : mfgpu_dropin::MFBase<Scalar>(3, A, Nx, Ny, Nz, width, maxSideLength) {}
};
}  // namespace TreeFactor3D

#endif
