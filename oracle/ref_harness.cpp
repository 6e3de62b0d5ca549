// Test infrastructure only: a driver around the UNMODIFIED reference
// (victorminden/updating-multifrontal) compiled from its own sources.
// It is never linked into the product.  It reads a problem description
// (coefficient field, options, right-hand sides) from a binary file, builds the
// matrix with the reference fixture (test_include/DE/buildLaplacian.hpp:10,244),
// runs MF2D/MF3D Factor / Update / Solve / Apply (include/DE/mf.hpp:67-80,173-188)
// and writes what it saw (CSR, per-level DOF lists, per-front dense blocks,
// solutions, timings) to a binary record file read by oracle/refio.py.
//
// Private members are reached with `#define private public` after all standard
// headers are included, so the reference headers stay untouched.

#include <algorithm>
#include <cassert>
#include <chrono>
#include <climits>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#define private public
#include "linalg.hpp"
#include "buildLaplacian.hpp"
#include "mf.hpp"
#undef private

using namespace LinAlg;

namespace {

struct Writer {
  FILE* f;
  explicit Writer(const char* path) { f = fopen(path, "wb"); if (!f) { perror(path); exit(2); } }
  ~Writer() { if (f) fclose(f); }
  void rec(const std::string& name, char dtype, const void* data, uint64_t count) {
    uint32_t nl = (uint32_t)name.size();
    fwrite(&nl, 4, 1, f);
    fwrite(name.data(), 1, nl, f);
    fwrite(&dtype, 1, 1, f);
    fwrite(&count, 8, 1, f);
    size_t es = dtype == 'd' ? 8 : 4;
    if (count) fwrite(data, es, count, f);
  }
  void ints(const std::string& n, const std::vector<int>& v) { rec(n, 'i', v.data(), v.size()); }
  void dbls(const std::string& n, const std::vector<double>& v) { rec(n, 'd', v.data(), v.size()); }
  void dense(const std::string& n, const Dense<double>& A) {
    std::vector<int> shape = {A.m(), A.n()};
    ints(n + ".shape", shape);
    if ((size_t)A.m() * A.n() > 0 && A.data_.size() >= (size_t)A.m() * A.n())
      rec(n, 'd', A.data_.data(), (uint64_t)A.m() * A.n());
    else
      rec(n, 'd', nullptr, 0);
  }
};

struct Input {
  int dim, Nx, Ny, Nz, width, maxSide;
  int dumpSymbolic, dumpFronts, doUpdate, nrhs, timeReps, solveReps;
  double hx, hy, hz;
  std::vector<double> coef1, coef2;
  std::vector<double> rhs;   // nrhs * n
};

Input readInput(const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  Input in;
  int32_t hdr[12];
  if (fread(hdr, 4, 12, f) != 12) { fprintf(stderr, "bad header\n"); exit(2); }
  in.dim = hdr[0]; in.Nx = hdr[1]; in.Ny = hdr[2]; in.Nz = hdr[3];
  in.width = hdr[4]; in.maxSide = hdr[5]; in.dumpSymbolic = hdr[6];
  in.dumpFronts = hdr[7]; in.doUpdate = hdr[8]; in.nrhs = hdr[9];
  in.timeReps = hdr[10]; in.solveReps = hdr[11];
  double h[3];
  if (fread(h, 8, 3, f) != 3) { fprintf(stderr, "bad h\n"); exit(2); }
  in.hx = h[0]; in.hy = h[1]; in.hz = h[2];
  size_t nc = (size_t)(in.Nx + 2 * in.width) * (in.Ny + 2 * in.width) *
              (in.dim == 3 ? (in.Nz + 2 * in.width) : 1);
  in.coef1.resize(nc);
  if (fread(in.coef1.data(), 8, nc, f) != nc) { fprintf(stderr, "bad coef1\n"); exit(2); }
  if (in.doUpdate) {
    in.coef2.resize(nc);
    if (fread(in.coef2.data(), 8, nc, f) != nc) { fprintf(stderr, "bad coef2\n"); exit(2); }
  }
  size_t n = (size_t)in.Nx * in.Ny * (in.dim == 3 ? in.Nz : 1);
  in.rhs.resize((size_t)in.nrhs * n);
  if (in.nrhs && fread(in.rhs.data(), 8, in.rhs.size(), f) != in.rhs.size()) {
    fprintf(stderr, "bad rhs\n"); exit(2);
  }
  fclose(f);
  return in;
}

SMat build2(const Input& in, const std::vector<double>& c) {
  int W = in.width, sx = in.Nx + 2 * W, sy = in.Ny + 2 * W;
  std::vector<std::vector<double> > A(sx, std::vector<double>(sy));
  for (int i = 0; i < sx; i++)
    for (int j = 0; j < sy; j++) A[i][j] = c[(size_t)i * sy + j];
  return buildLaplacian(in.Nx, in.Ny, A, W, in.hx, in.hy);
}

SMat build3(const Input& in, const std::vector<double>& c) {
  int W = in.width, sx = in.Nx + 2 * W, sy = in.Ny + 2 * W, sz = in.Nz + 2 * W;
  std::vector<std::vector<std::vector<double> > > A(
      sx, std::vector<std::vector<double> >(sy, std::vector<double>(sz)));
  for (int i = 0; i < sx; i++)
    for (int j = 0; j < sy; j++)
      for (int k = 0; k < sz; k++) A[i][j][k] = c[((size_t)i * sy + j) * sz + k];
  return buildLaplacian(in.Nx, in.Ny, in.Nz, A, W, in.hx, in.hy, in.hz);
}

void dumpCSR(Writer& w, const std::string& p, SMat& M) {
  w.ints(p + "row_ptr", M.row_ptr_);
  w.ints(p + "col_ind", M.col_ind_);
  w.dbls(p + "val", M.val_);
}

// Modified DOFs exactly as test_src/DE/testMF2D.cpp:143-150 computes them.
std::set<int> diffDOFs(SMat& M1, SMat& M2) {
  std::set<int> mod;
  for (int idx = 0; idx < M1.nnz(); idx++)
    if (M1.val(idx) != M2.val(idx)) mod.insert(M1.col_ind(idx));
  return mod;
}

double secs(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

template <class MF, class SepVec>
void dumpTree(Writer& w, MF& F, std::vector<std::vector<SepVec> >& seps, bool fronts) {
  std::vector<int> lv = {F.levels_};
  w.ints("levels", lv);
  for (int ell = 0; ell < F.levels_; ell++) {
    auto& boxes = F.boxData_[ell];
    for (size_t b = 0; b < boxes.size(); b++) {
      std::string p = "box." + std::to_string(ell) + "." + std::to_string(b) + ".";
      w.ints(p + "int", boxes[b].intDOFs);
      w.ints(p + "bd", boxes[b].bdDOFs);
      if (fronts) {
        w.dense(p + "A22", boxes[b].A22);
        w.dense(p + "XL", boxes[b].XL);
        w.dense(p + "XR", boxes[b].XR);
        w.dense(p + "S", boxes[b].SchurComp);
        w.dense(p + "A11post", boxes[b].A11post);
      }
    }
  }
  for (size_t l = 0; l < seps.size(); l++) {
    for (size_t e = 0; e < seps[l].size(); e++) {
      // separator storage index l holds the separators of box level l+1
      std::string p = "sep." + std::to_string(l + 1) + "." + std::to_string(e) + ".";
      w.ints(p + "dofs", seps[l][e].DOFs);
      if (fronts) w.dense(p + "A11", seps[l][e].A11);
    }
  }
}

template <class MF>
void runSolves(Writer& w, MF& F, SMat& M, const Input& in, size_t n, const std::string& tag) {
  for (int r = 0; r < in.nrhs; r++) {
    Vec<double> b((int)n);
    for (size_t i = 0; i < n; i++) b(i) = in.rhs[(size_t)r * n + i];
    Vec<double> x = F.Solve(b);
    Vec<double> y = F.Apply(b);
    std::vector<double> xs(x.data_.begin(), x.data_.end());
    std::vector<double> ys(y.data_.begin(), y.data_.end());
    w.dbls(tag + "solve." + std::to_string(r), xs);
    w.dbls(tag + "apply." + std::to_string(r), ys);
    Vec<double> Ax = M * x;
    Ax -= b;
    std::vector<double> res = {Ax.norm() / b.norm()};
    w.dbls(tag + "resid." + std::to_string(r), res);
  }
}

template <class MF, class SepGetter>
int runAll(const Input& in, const char* outPath, SMat M1, SMat M2, MF* F, SepGetter seps) {
  Writer w(outPath);
  size_t n = (size_t)M1.m();
  dumpCSR(w, "A1.", M1);
  auto t0 = std::chrono::steady_clock::now();
  F->Factor();
  auto t1 = std::chrono::steady_clock::now();
  std::vector<double> tf = {secs(t0, t1)};
  w.dbls("time.factor", tf);
  if (in.dumpSymbolic) dumpTree(w, *F, seps(*F), in.dumpFronts != 0);
  runSolves(w, *F, M1, in, n, "f1.");
  if (in.doUpdate) {
    dumpCSR(w, "A2.", M2);
    std::set<int> mod = diffDOFs(M1, M2);
    std::vector<int> modv(mod.begin(), mod.end());
    w.ints("moddofs", modv);
    auto t2 = std::chrono::steady_clock::now();
    F->Update(M2, mod);
    auto t3 = std::chrono::steady_clock::now();
    std::vector<double> tu = {secs(t2, t3)};
    w.dbls("time.update", tu);
    if (in.dumpSymbolic) dumpTree(w, *F, seps(*F), in.dumpFronts != 0);
    runSolves(w, *F, M2, in, n, "f2.");
  }
  return 0;
}

// Algorithmic work of the timed calls, counted from the reference's own front
// sizes after Factor (n = |intDOFs|, m = |bdDOFs| of every box) in the
// Cholesky form the GPU path reports: factor sum(n^3/3 + n^2 m + n m^2), solve
// sum 2(n^2 + 2 n m) per right-hand side, update the factor sum over the root
// paths of the leaves that Update() marks (the leaf of a DOF by the integer
// division of src/DE/mf2d.cpp:163-174 / mf3d.cpp:223-240, clamped to the last
// box; parents by the reference's getParentIdxFromBoxIdx_).
struct Work {
  double factor = 0, update = 0, solve_per_rhs = 0;
  long fronts = 0, dirty = 0;
};

double frontFlops(double n, double m) { return n * n * n / 3.0 + n * n * m + n * m * m; }

template <class MF, class LeafOf, class ParentOf>
Work workOf(MF& F, const std::set<int>& mod, LeafOf leafOf, ParentOf parentOf) {
  Work w;
  for (int ell = 0; ell < F.levels_; ell++)
    for (auto& b : F.boxData_[ell]) {
      const double n = (double)b.intDOFs.size(), m = (double)b.bdDOFs.size();
      w.factor += frontFlops(n, m);
      w.solve_per_rhs += 2.0 * (n * n + 2.0 * n * m);
      w.fronts++;
    }
  std::set<int> marked;
  for (int d : mod) marked.insert(leafOf(d));
  for (int ell = F.levels_ - 1; ell >= 0 && !marked.empty(); ell--) {
    std::set<int> up;
    for (int b : marked) {
      auto& box = F.boxData_[ell][b];
      w.update += frontFlops((double)box.intDOFs.size(), (double)box.bdDOFs.size());
      w.dirty++;
      if (ell > 0) up.insert(parentOf(b, ell));
    }
    marked.swap(up);
  }
  return w;
}

Work work2(TreeFactor2D::MF2D<double>& F, const std::set<int>& mod) {
  const int bps = 1 << (F.levels_ - 1);
  auto leaf = [&](int idx) {
    const int i = idx % F.Nx_, j = idx / F.Nx_;
    const int ib = std::min(i / (F.boxWidthXBottom_ + F.width_), bps - 1);
    const int jb = std::min(j / (F.boxWidthYBottom_ + F.width_), bps - 1);
    return TreeFactor2D::TensorIdx2D(ib, jb, bps, bps).LinearIndex();
  };
  return workOf(F, mod, leaf, [](int b, int ell) { return TreeFactor2D::getParentIdxFromBoxIdx_(b, ell); });
}

Work work3(TreeFactor3D::MF3D<double>& F, const std::set<int>& mod) {
  const int bps = 1 << (F.levels_ - 1);
  auto leaf = [&](int idx) {
    const int i = idx % F.Nx_, j = (idx / F.Nx_) % F.Ny_, k = idx / F.Nx_ / F.Ny_;
    const int ib = std::min(i / (F.boxWidthXBottom_ + F.width_), bps - 1);
    const int jb = std::min(j / (F.boxWidthYBottom_ + F.width_), bps - 1);
    const int kb = std::min(k / (F.boxWidthZBottom_ + F.width_), bps - 1);
    return TreeFactor3D::TensorIdx3D(ib, jb, kb, bps, bps, bps).LinearIndex();
  };
  return workOf(F, mod, leaf, [](int b, int ell) { return TreeFactor3D::getParentIdxFromBoxIdx_(b, ell); });
}

Work workFor(TreeFactor2D::MF2D<double>& F, const std::set<int>& mod) { return work2(F, mod); }
Work workFor(TreeFactor3D::MF3D<double>& F, const std::set<int>& mod) { return work3(F, mod); }

// Timing mode for the CPU baseline: repeated Factor, Update, Solve on the same
// inputs, one JSON line on stdout (seconds per call and the work figures).
template <class MF>
int runTiming(const Input& in, SMat& M1, SMat& M2, MF* F) {
  size_t n = (size_t)M1.m();
  std::set<int> mod;
  if (in.doUpdate) mod = diffDOFs(M1, M2);
  std::vector<double> tf, tu, ts;
  Vec<double> b((int)n);
  for (size_t i = 0; i < n; i++) b(i) = in.nrhs ? in.rhs[i] : 1.0;
  std::set<int> all;
  for (size_t i = 0; i < n; i++) all.insert((int)i);
  Work work;
  for (int r = 0; r < std::max(1, in.timeReps); r++) {
    auto a = std::chrono::steady_clock::now();
    if (r > 0) {
      // Factor() marks only what the previous call left marked, so a repeat
      // refactors from scratch through Update() with every DOF modified.
      F->Update(M1, all);
    } else {
      F->Factor();
    }
    auto bt = std::chrono::steady_clock::now();
    tf.push_back(secs(a, bt));
    if (r == 0) work = workFor(*F, mod);
    if (in.doUpdate) {
      auto c = std::chrono::steady_clock::now();
      F->Update(M2, mod);
      auto d = std::chrono::steady_clock::now();
      tu.push_back(secs(c, d));
    }
    for (int s = 0; s < std::max(1, in.solveReps); s++) {
      auto e = std::chrono::steady_clock::now();
      for (int k = 0; k < std::max(1, in.nrhs); k++) {
        Vec<double> x = F->Solve(b);
        (void)x;
      }
      auto g = std::chrono::steady_clock::now();
      ts.push_back(secs(e, g));
    }
  }
  auto js = [](const std::vector<double>& v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); i++) {
      char buf[64];
      snprintf(buf, sizeof buf, "%s%.9g", i ? ", " : "", v[i]);
      s += buf;
    }
    return s + "]";
  };
  printf("{\"factor_s\": %s, \"update_s\": %s, \"solve_s\": %s, \"factor_flops\": %.9g, "
         "\"update_flops\": %.9g, \"solve_flops_per_rhs\": %.9g, \"fronts\": %ld, "
         "\"dirty_fronts\": %ld, \"n\": %zu, \"nnz\": %d}\n",
         js(tf).c_str(), js(tu).c_str(), js(ts).c_str(), work.factor, work.update,
         work.solve_per_rhs, work.fronts, work.dirty, n, M1.nnz());
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s dump|time|csr input.bin output.bin\n", argv[0]);
    return 2;
  }
  std::string mode = argv[1];
  Input in = readInput(argv[2]);
  try {
    if (mode == "csr") {   // only the fixture's CSR (buildLaplacian.hpp), no factorization
      SMat M1 = in.dim == 2 ? build2(in, in.coef1) : build3(in, in.coef1);
      Writer w(argv[3]);
      dumpCSR(w, "A1.", M1);
      return 0;
    }
    if (in.dim == 2) {
      SMat M1 = build2(in, in.coef1);
      SMat M2 = in.doUpdate ? build2(in, in.coef2) : M1;
      TreeFactor2D::MF2D<double> F(M1, in.Nx, in.Ny, in.width, in.maxSide);
      if (mode == "time") return runTiming(in, M1, M2, &F);
      return runAll(in, argv[3], M1, M2, &F,
                    [](TreeFactor2D::MF2D<double>& G) -> decltype(G.edgeData_)& { return G.edgeData_; });
    } else {
      SMat M1 = build3(in, in.coef1);
      SMat M2 = in.doUpdate ? build3(in, in.coef2) : M1;
      TreeFactor3D::MF3D<double> F(M1, in.Nx, in.Ny, in.Nz, in.width, in.maxSide);
      if (mode == "time") return runTiming(in, M1, M2, &F);
      return runAll(in, argv[3], M1, M2, &F,
                    [](TreeFactor3D::MF3D<double>& G) -> decltype(G.faceData_)& { return G.faceData_; });
    }
  } catch (const std::exception& e) {
    fprintf(stderr, "reference threw: %s\n", e.what());
    return 3;
  }
}
