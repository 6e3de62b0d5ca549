// Drop-in check, written like the reference's own drivers
// (test_src/DE/testMF2D.cpp:124-278, testMF3D.cpp:137-289): a caller that only
// includes linalg.hpp and mf.hpp factors, applies, solves and updates through
// TreeFactor2D::MF2D / TreeFactor3D::MF3D.  Exit status 0 when every error is
// at rounding level and the stale factor's apply error is large.
#include <cmath>
#include <cstdio>
#include <random>
#include <set>
#include <stdexcept>
#include <vector>

#include "laplacian.hpp"
#include "linalg.hpp"
#include "mf.hpp"

using LinAlg::Sparse;
using LinAlg::Vec;

static int failures = 0;
static void expect(bool ok, const char* what, double v) {
  std::printf("%-48s %.3e %s\n", what, v, ok ? "ok" : "FAIL");
  if (!ok) failures++;
}

static std::set<int> modified(Sparse<double>& M1, Sparse<double>& M2) {
  std::set<int> mod;   // testMF2D.cpp:143-150
  for (int idx = 0; idx < M1.nnz(); idx++)
    if (M1.val(idx) != M2.val(idx)) mod.insert(M1.col_ind(idx));
  return mod;
}

static Vec<double> randomVec(int n, unsigned seed) {
  std::mt19937 g(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  Vec<double> x(n);
  for (int i = 0; i < n; i++) x(i) = u(g);
  return x;
}

static void test2D(int N, int maxSide) {
  std::vector<std::vector<double> > a(N + 2, std::vector<double>(N + 2, 1.0)), a2 = a;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) a2[i][j] *= 2;
  Sparse<double> M1 = laplacian2D(N, N, a), M2 = laplacian2D(N, N, a2);
  Vec<double> x = randomVec(N * N, 1234);
  Vec<double> b1 = M1 * x;
  TreeFactor2D::MF2D<double> F(M1, N, N, 1, maxSide);
  F.Factor();
  Vec<double> r = F.Apply(x);
  r -= b1;
  expect(r.norm() / b1.norm() < 1e-14, "2D relative apply error", r.norm() / b1.norm());
  Vec<double> y = F.Solve(b1);
  y -= x;
  expect(y.norm() / x.norm() < 1e-11, "2D relative solve error", y.norm() / x.norm());
  Vec<double> btrue = M2 * x;
  Vec<double> s1 = F.Apply(x);
  s1 -= btrue;
  F.Update(M2, modified(M1, M2));
  Vec<double> s2 = F.Apply(x);
  s2 -= btrue;
  expect(s1.norm() / btrue.norm() > 1e-4, "2D apply error without updating", s1.norm() / btrue.norm());
  expect(s2.norm() / btrue.norm() < 1e-14, "2D apply error after updating", s2.norm() / btrue.norm());
}

static void test3D(int N, int maxSide) {
  std::vector<std::vector<std::vector<double> > > a(
      N + 2, std::vector<std::vector<double> >(N + 2, std::vector<double>(N + 2, 1.0)));
  std::mt19937 g(7);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  for (auto& p : a)
    for (auto& q : p)
      for (double& c : q) c = 1.0 + u(g);   // testMF3D.cpp:89-106: 1 + rand
  auto a2 = a;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) a2[i][j][k] *= 2;
  Sparse<double> M1 = laplacian3D(N, N, N, a), M2 = laplacian3D(N, N, N, a2);
  Vec<double> x = randomVec(N * N * N, 99);
  Vec<double> b1 = M1 * x;
  TreeFactor3D::MF3D<double> F(M1, N, N, N, 1, maxSide);
  F.Factor();
  Vec<double> r = F.Apply(x);
  r -= b1;
  expect(r.norm() / b1.norm() < 1e-14, "3D relative apply error", r.norm() / b1.norm());
  Vec<double> y = F.Solve(b1);
  y -= x;
  expect(y.norm() / x.norm() < 1e-12, "3D relative solve error", y.norm() / x.norm());
  Vec<double> btrue = M2 * x;
  F.Update(M2, modified(M1, M2));
  Vec<double> s2 = F.Apply(x);
  s2 -= btrue;
  expect(s2.norm() / btrue.norm() < 1e-14, "3D apply error after updating", s2.norm() / btrue.norm());
}

int main() {
  test2D(127, 8);
  test3D(31, 4);
  // the reference's error behaviour: too shallow a tree throws runtime_error
  bool threw = false;
  try {
    std::vector<std::vector<double> > a(33, std::vector<double>(33, 1.0));
    Sparse<double> M = laplacian2D(31, 31, a);
    TreeFactor2D::MF2D<double> F(M, 31, 31, 1, 40);
  } catch (const std::runtime_error&) {
    threw = true;
  }
  expect(threw, "depth-1 tree throws std::runtime_error", threw ? 1.0 : 0.0);
  std::printf("%s\n", failures ? "FAILED" : "PASSED");
  return failures ? 1 : 0;
}
