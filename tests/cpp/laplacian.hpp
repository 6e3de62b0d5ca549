// Test fixture: variable-coefficient 5-point (2D) / 7-point (3D) Laplacian,
// separator width 1, restating the reference fixture
// (test_include/DE/buildLaplacian.hpp:10-132, 244-391): node coefficients
// indexed A[i][j](k) with one ghost layer, face value = mean of its two nodes,
// off-diagonal -a/h^2, diagonal the sum of the face terms, columns ascending.
#pragma once
#include <vector>

#include "linalg.hpp"

inline LinAlg::Sparse<double> laplacian2D(int Nx, int Ny, const std::vector<std::vector<double> >& A) {
  IdxVec rp, ci;
  std::vector<double> v;
  int off = 0;
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nx; i++) {
      rp.push_back(off);
      const int ii = i + 1, jj = j + 1, idx = i + j * Nx;
      auto push = [&](int c, double x) { ci.push_back(c); v.push_back(x); off++; };
      if (j - 1 >= 0) push(idx - Nx, -1.0 * (0.5 * (A[ii][jj - 1] + A[ii][jj])));
      if (i - 1 >= 0) push(idx - 1, -1.0 * (0.5 * (A[ii - 1][jj] + A[ii][jj])));
      double d = 0;
      d -= -1.0 * (0.5 * (A[ii - 1][jj] + A[ii][jj]) + 0.5 * (A[ii + 1][jj] + A[ii][jj]));
      d -= -1.0 * (0.5 * (A[ii][jj - 1] + A[ii][jj]) + 0.5 * (A[ii][jj + 1] + A[ii][jj]));
      push(idx, d);
      if (i + 1 <= Nx - 1) push(idx + 1, -1.0 * (0.5 * (A[ii + 1][jj] + A[ii][jj])));
      if (j + 1 <= Ny - 1) push(idx + Nx, -1.0 * (0.5 * (A[ii][jj + 1] + A[ii][jj])));
    }
  rp.push_back(off);
  return LinAlg::Sparse<double>(v, ci, rp, Nx * Ny, Nx * Ny);
}

inline LinAlg::Sparse<double> laplacian3D(int Nx, int Ny, int Nz,
                                          const std::vector<std::vector<std::vector<double> > >& A) {
  IdxVec rp, ci;
  std::vector<double> v;
  int off = 0;
  const int sxy = Nx * Ny;
  for (int z = 0; z < Nz; z++)
    for (int j = 0; j < Ny; j++)
      for (int i = 0; i < Nx; i++) {
        rp.push_back(off);
        const int ii = i + 1, jj = j + 1, zz = z + 1, idx = i + j * Nx + z * sxy;
        auto push = [&](int c, double x) { ci.push_back(c); v.push_back(x); off++; };
        const double c = A[ii][jj][zz];
        if (z - 1 >= 0) push(idx - sxy, -1.0 * (0.5 * (A[ii][jj][zz - 1] + c)));
        if (j - 1 >= 0) push(idx - Nx, -1.0 * (0.5 * (A[ii][jj - 1][zz] + c)));
        if (i - 1 >= 0) push(idx - 1, -1.0 * (0.5 * (A[ii - 1][jj][zz] + c)));
        double d = 0;
        d -= -1.0 * (0.5 * (A[ii - 1][jj][zz] + c) + 0.5 * (A[ii + 1][jj][zz] + c));
        d -= -1.0 * (0.5 * (A[ii][jj - 1][zz] + c) + 0.5 * (A[ii][jj + 1][zz] + c));
        d -= -1.0 * (0.5 * (A[ii][jj][zz - 1] + c) + 0.5 * (A[ii][jj][zz + 1] + c));
        push(idx, d);
        if (i + 1 <= Nx - 1) push(idx + 1, -1.0 * (0.5 * (A[ii + 1][jj][zz] + c)));
        if (j + 1 <= Ny - 1) push(idx + Nx, -1.0 * (0.5 * (A[ii][jj + 1][zz] + c)));
        if (z + 1 <= Nz - 1) push(idx + sxy, -1.0 * (0.5 * (A[ii][jj][zz + 1] + c)));
      }
  rp.push_back(off);
  return LinAlg::Sparse<double>(v, ci, rp, Nx * Ny * Nz, Nx * Ny * Nz);
}
