#include "schedule.hpp"

#include <algorithm>
#include <array>
#include <climits>

#include <algorithm>
#include <cmath>
#include <set>
#include <stdexcept>

namespace mfgpu {

namespace {
enum { L2R = 0, T2B = 1 };
enum { XN = 0, YN = 1, ZN = 2 };

// ---- 2D topology (src/DE/tree2d_common.cpp) ----
int edgeType(int e, int ell) {                      // tree2d_common.cpp:8-11
  int bps = 1 << ell;
  return (e % (2 * bps - 1)) < bps - 1 ? T2B : L2R;
}
int edgeIdx(int row, int col, int ell, int type) {  // tree2d_common.cpp:15-26
  int bps = 1 << ell;
  return type == L2R ? row * (2 * bps - 1) + col + bps - 1 : row * (2 * bps - 1) + col;
}
void edgeCoords(int e, int ell, int& x, int& y) {   // tree2d_common.cpp:28-35
  int bps = 1 << ell;
  if (edgeType(e, ell) == L2R) e -= bps - 1;
  int w = 2 * bps - 1;
  x = e % w;
  y = e / w;
}
// ---- 3D topology (src/DE/tree3d_common.cpp) ----
int faceType(int f, int ell) {                      // tree3d_common.cpp:9-19
  int bps = 1 << ell;
  int fps = 2 * (bps - 1) * bps + bps * bps;
  f %= fps;
  if (f >= 2 * (bps - 1) * bps) return ZN;
  f %= 2 * bps - 1;
  return f < bps - 1 ? XN : YN;
}
int faceIdx(int row, int col, int sli, int ell, int type) {  // tree3d_common.cpp:23-40
  int bps = 1 << ell;
  int fps = 2 * (bps - 1) * bps + bps * bps;
  if (type == XN) return sli * fps + row * (2 * bps - 1) + col;
  if (type == YN) return sli * fps + row * (2 * bps - 1) + col + bps - 1;
  return sli * fps + row * bps + col + 2 * (bps - 1) * bps;
}
void faceCoords(int f, int ell, int& x, int& y, int& z) {     // tree3d_common.cpp:43-71
  int bps = 1 << ell;
  int fps = 2 * (bps - 1) * bps + bps * bps;
  int t = faceType(f, ell);
  if (t == ZN) {
    f -= 2 * (bps - 1) * bps;
    z = f / fps;
    f -= z * fps;
    y = f / bps;
    x = f - y * bps;
    return;
  }
  if (t == YN) f -= bps - 1;
  z = f / fps;
  f -= z * fps;
  y = f / (2 * bps - 1);
  x = f - y * (2 * bps - 1);
}
inline int64_t roundUp(int64_t v, int64_t a) { return (v + a - 1) / a * a; }
}  // namespace

int Schedule::nboxAt(int ell) const {
  int bps = 1 << ell;
  return dim == 2 ? bps * bps : bps * bps * bps;
}
int Schedule::nsepAt(int ell) const {
  int bps = 1 << ell;
  return dim == 2 ? 2 * bps * bps - 2 * bps : 3 * bps * bps * (bps - 1);
}

std::vector<int> Schedule::nborSeps(int b, int ell) const {
  int bps = 1 << ell;
  if (dim == 2) {                                   // tree2d_common.cpp:135-184
    int x = b % bps, y = b / bps;
    return {x > 0 ? edgeIdx(y, x - 1, ell, T2B) : -1, x < bps - 1 ? edgeIdx(y, x, ell, T2B) : -1,
            y > 0 ? edgeIdx(y - 1, x, ell, L2R) : -1, y < bps - 1 ? edgeIdx(y, x, ell, L2R) : -1};
  }
  int x = b % bps, y = (b / bps) % bps, z = b / (bps * bps);  // tree3d_common.cpp:185-275
  return {x > 0 ? faceIdx(y, x - 1, z, ell, XN) : -1, x < bps - 1 ? faceIdx(y, x, z, ell, XN) : -1,
          y > 0 ? faceIdx(y - 1, x, z, ell, YN) : -1, y < bps - 1 ? faceIdx(y, x, z, ell, YN) : -1,
          z > 0 ? faceIdx(y, x, z - 1, ell, ZN) : -1, z < bps - 1 ? faceIdx(y, x, z, ell, ZN) : -1};
}

void Schedule::nborBoxes(int e, int ell, int out[2]) const {
  int bps = 1 << ell;
  if (dim == 2) {                                   // tree2d_common.cpp:186-211
    int x, y;
    edgeCoords(e, ell, x, y);
    out[0] = x + y * bps;
    out[1] = edgeType(e, ell) == T2B ? (x + 1) + y * bps : x + (y + 1) * bps;
    return;
  }
  int x, y, z;                                      // tree3d_common.cpp:277-312
  faceCoords(e, ell, x, y, z);
  int t = faceType(e, ell);
  out[0] = x + y * bps + z * bps * bps;
  if (t == XN) out[1] = (x + 1) + y * bps + z * bps * bps;
  else if (t == YN) out[1] = x + (y + 1) * bps + z * bps * bps;
  else out[1] = x + y * bps + (z + 1) * bps * bps;
}

std::vector<int> Schedule::childSeps(int e, int ell) const {
  if (dim == 2) {                                   // tree2d_common.cpp:91-119
    int x, y;
    edgeCoords(e, ell, x, y);
    if (edgeType(e, ell) == L2R)
      return {edgeIdx(2 * y + 1, 2 * x, ell + 1, L2R), edgeIdx(2 * y + 1, 2 * x + 1, ell + 1, L2R)};
    return {edgeIdx(2 * y, 2 * x + 1, ell + 1, T2B), edgeIdx(2 * y + 1, 2 * x + 1, ell + 1, T2B)};
  }
  int x, y, z;                                      // tree3d_common.cpp:127-164
  faceCoords(e, ell, x, y, z);
  int r = y, c = x, s = z, t = faceType(e, ell);
  if (t == XN)
    return {faceIdx(2 * r, 2 * c + 1, 2 * s, ell + 1, XN), faceIdx(2 * r, 2 * c + 1, 2 * s + 1, ell + 1, XN),
            faceIdx(2 * r + 1, 2 * c + 1, 2 * s, ell + 1, XN),
            faceIdx(2 * r + 1, 2 * c + 1, 2 * s + 1, ell + 1, XN)};
  if (t == YN)
    return {faceIdx(2 * r + 1, 2 * c, 2 * s, ell + 1, YN), faceIdx(2 * r + 1, 2 * c, 2 * s + 1, ell + 1, YN),
            faceIdx(2 * r + 1, 2 * c + 1, 2 * s, ell + 1, YN),
            faceIdx(2 * r + 1, 2 * c + 1, 2 * s + 1, ell + 1, YN)};
  return {faceIdx(2 * r, 2 * c, 2 * s + 1, ell + 1, ZN), faceIdx(2 * r + 1, 2 * c, 2 * s + 1, ell + 1, ZN),
          faceIdx(2 * r, 2 * c + 1, 2 * s + 1, ell + 1, ZN),
          faceIdx(2 * r + 1, 2 * c + 1, 2 * s + 1, ell + 1, ZN)};
}

std::vector<int> Schedule::childBoxes(int b, int ell) const {
  int bps = 1 << ell, c = 2 * bps;
  if (dim == 2) {                                   // tree2d_common.cpp:121-131
    int x = b % bps, y = b / bps;
    return {2 * x + 2 * y * c, 2 * x + (2 * y + 1) * c, (2 * x + 1) + 2 * y * c,
            (2 * x + 1) + (2 * y + 1) * c};
  }
  int x = b % bps, y = (b / bps) % bps, z = b / (bps * bps);  // tree3d_common.cpp:166-181
  static const int o[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                              {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  std::vector<int> r(8);
  for (int i = 0; i < 8; i++)
    r[i] = (2 * x + o[i][0]) + (2 * y + o[i][1]) * c + (2 * z + o[i][2]) * c * c;
  return r;
}

// Child separators interior to box b (tree2d_common.cpp:59-79,
// tree3d_common.cpp:95-115): those whose normal coordinate is even.
std::vector<int> Schedule::selfChildren(int b, int ell) const {
  std::set<int> s;
  for (int c : childBoxes(b, ell))
    for (int e : nborSeps(c, ell + 1)) {
      if (e == -1) continue;
      bool interior;
      if (dim == 2) {
        int x, y;
        edgeCoords(e, ell + 1, x, y);
        int t = edgeType(e, ell + 1);
        interior = (t == T2B && x % 2 == 0) || (t == L2R && y % 2 == 0);
      } else {
        int x, y, z;
        faceCoords(e, ell + 1, x, y, z);
        int t = faceType(e, ell + 1);
        interior = (t == XN && x % 2 == 0) || (t == YN && y % 2 == 0) || (t == ZN && z % 2 == 0);
      }
      if (interior) s.insert(e);
    }
  return std::vector<int>(s.begin(), s.end());
}

int Schedule::bwidth(int ell, int axis, bool below) const {
  int d = levels - 1 - ell - (below ? 1 : 0);
  return bw[axis] * (1 << d) + ((1 << d) - 1) * width;
}

void Schedule::block(const int lo[3], const int hi[3], std::vector<int>& out) const {
  int64_t sxy = (int64_t)N[0] * N[1];
  int zl = dim == 3 ? lo[2] : 0, zh = dim == 3 ? hi[2] : 1;
  for (int k = zl; k < zh; k++)
    for (int j = lo[1]; j < hi[1]; j++)
      for (int i = lo[0]; i < hi[0]; i++) out.push_back((int)(i + (int64_t)j * N[0] + k * sxy));
}

// mf2d.cpp:186-218, mf3d.cpp:253-348
std::vector<int> Schedule::boxCenters(int b, int ell) const {
  int bps = 1 << ell, w = width;
  int BW[3], BB[3], c[3];
  for (int a = 0; a < dim; a++) {
    BW[a] = bwidth(ell, a, false);
    BB[a] = bwidth(ell, a, true);
  }
  c[0] = b % bps;
  c[1] = (b / bps) % bps;
  c[2] = dim == 3 ? b / (bps * bps) : 0;
  std::vector<int> out;
  if (dim == 2) {
    int lo[3] = {c[0] * (BW[0] + w) + BB[0], c[1] * (BW[1] + w) + BB[1], 0};
    int hi[3] = {lo[0] + w, lo[1] + w, 1};
    block(lo, hi, out);
    return out;
  }
  for (int axis = 0; axis < 3; axis++) {
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      if (a == axis) {
        lo[a] = c[a] * (BW[a] + w);
        hi[a] = c[a] == bps - 1 ? N[a] : lo[a] + BW[a];
      } else {
        lo[a] = c[a] * (BW[a] + w) + BB[a];
        hi[a] = lo[a] + w;
      }
    }
    block(lo, hi, out);
  }
  std::sort(out.begin(), out.end());            // the reference collects a std::set
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// mf2d.cpp:220-270, mf3d.cpp:350-524
std::vector<int> Schedule::sepCenters(int e, int ell) const {
  int bps = 1 << ell, w = width;
  int BW[3], BB[3];
  for (int a = 0; a < dim; a++) {
    BW[a] = bwidth(ell, a, false);
    BB[a] = bwidth(ell, a, true);
  }
  std::vector<int> out;
  if (dim == 2) {
    int x, y;
    edgeCoords(e, ell, x, y);
    int lo[3];
    if (edgeType(e, ell) == L2R) {
      lo[0] = x * (BW[0] + w) + BB[0];
      lo[1] = y * (BW[1] + w) + BW[1];
    } else {
      lo[0] = x * (BW[0] + w) + BW[0];
      lo[1] = y * (BW[1] + w) + BB[1];
    }
    lo[2] = 0;
    int hi[3] = {lo[0] + w, lo[1] + w, 1};
    block(lo, hi, out);
    return out;
  }
  int c[3];
  faceCoords(e, ell, c[0], c[1], c[2]);
  int normal = faceType(e, ell);  // XN=0, YN=1, ZN=2 match the axis numbers
  for (int axis = 0; axis < 3; axis++) {
    if (axis == normal) continue;
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      if (a == normal) {
        lo[a] = c[a] * (BW[a] + w) + BW[a];
        hi[a] = lo[a] + w;
      } else if (a == axis) {
        lo[a] = c[a] * (BW[a] + w);
        hi[a] = c[a] == bps - 1 ? N[a] : lo[a] + BW[a];
      } else {
        lo[a] = c[a] * (BW[a] + w) + BB[a];
        hi[a] = lo[a] + w;
      }
    }
    block(lo, hi, out);
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

Schedule::Schedule(int dim_, int nx, int ny, int nz, int width_, int max_side, bool full_storage_)
    : dim(dim_), width(width_), full_storage(full_storage_) {
  if (dim != 2 && dim != 3) throw std::invalid_argument("dim must be 2 or 3");
  N[0] = nx;
  N[1] = ny;
  N[2] = dim == 3 ? nz : 1;
  if (nx <= 0 || ny <= 0 || (dim == 3 && nz <= 0) || width <= 0 || max_side <= 0)
    throw std::invalid_argument("grid sizes, width and maxSideLength must be positive");
  ndof = (int64_t)N[0] * N[1] * N[2];
  if (ndof > 0x7fffffffLL) throw std::invalid_argument("more than 2^31-1 DOFs");
  // tree depth (mf2d.cpp:23-31, mf3d.cpp:41-51)
  int top = std::max(N[0], N[1]);
  if (dim == 3) top = std::max(top, N[2]);
  double num = top + width, den = max_side + width;
  levels = (int)std::ceil(std::log2(num / den));
  if (levels <= 1)
    throw std::runtime_error(
        "Based on the input parameters, the recursion depth is 1 level (i.e., do not recurse).  "
        "Try increasing the problem size or decreasing maxSideLength.");
  int bps = 1 << (levels - 1);
  for (int a = 0; a < dim; a++) {
    bw[a] = (int)std::floor((double)(N[a] - (bps - 1) * width) / (double)bps);
    if (N[a] < bw[a] * (bps - 1) + width * (bps - 1))
      throw std::runtime_error(
          "You found a bug!  The math for computing the number of points per box at a leaf "
          "level broke on this input.");
    if (bw[a] <= 0)
      throw std::runtime_error("leaf boxes would be empty: decrease the tree depth");
  }
  if (dim == 2) bw[2] = 1;
  B_.resize(levels);
  S_.resize(levels);
  for (int ell = 0; ell < levels; ell++) {
    B_[ell].resize(nboxAt(ell));
    if (ell >= 1) S_[ell].resize(nsepAt(ell));
  }
  buildLeaves();
  buildUpper();
  layout();
  buildTasks();
  B_.clear();
  S_.clear();
}

// mf2d.cpp:73-133, mf3d.cpp:96-188
void Schedule::buildLeaves() {
  int ell = levels - 1, bps = 1 << ell, w = width;
  int nb = nboxAt(ell);
  for (int b = 0; b < nb; b++) {
    int c[3] = {b % bps, (b / bps) % bps, dim == 3 ? b / (bps * bps) : 0};
    int first[3], ub[3];
    for (int a = 0; a < 3; a++) {
      if (a < dim) {
        first[a] = c[a] * (bw[a] + w);
        ub[a] = c[a] == bps - 1 ? N[a] : first[a] + bw[a];
      } else {
        first[a] = 0;
        ub[a] = 1;
      }
    }
    BoxSym& box = B_[ell][b];
    block(first, ub, box.piv);
    std::vector<int> ns = nborSeps(b, ell);
    // each separator is filled by one adjacent box: left (slot 0) and top
    // (slot 3) in 2D, plus below (slot 4) in 3D.
    if (c[0] > 0) {
      int lo[3] = {first[0] - w, first[1], first[2]}, hi[3] = {first[0], ub[1], ub[2]};
      block(lo, hi, S_[ell][ns[0]].dofs);
    }
    if (c[1] < bps - 1) {
      int lo[3] = {first[0], ub[1], first[2]}, hi[3] = {ub[0], ub[1] + w, ub[2]};
      block(lo, hi, S_[ell][ns[3]].dofs);
    }
    if (dim == 3 && c[2] > 0) {
      int lo[3] = {first[0], first[1], first[2] - w}, hi[3] = {ub[0], ub[1], first[2]};
      block(lo, hi, S_[ell][ns[4]].dofs);
    }
  }
  for (int b = 0; b < nb; b++) {
    BoxSym& box = B_[ell][b];
    box.nbseps = nborSeps(b, ell);
    for (int e : box.nbseps) {
      box.bdoff.push_back(e == -1 ? -1 : (int)box.bd.size());
      if (e != -1) box.bd.insert(box.bd.end(), S_[ell][e].dofs.begin(), S_[ell][e].dofs.end());
    }
  }
}

// mf2d.cpp:274-446, mf3d.cpp:528-702 (symbolic part)
void Schedule::buildUpper() {
  for (int ell = levels - 2; ell >= 0; ell--) {
    if (ell >= 1) {
      for (int e = 0; e < nsepAt(ell); e++) {
        SepSym& s = S_[ell][e];
        s.kids = childSeps(e, ell);
        for (int c : s.kids) s.dofs.insert(s.dofs.end(), S_[ell + 1][c].dofs.begin(), S_[ell + 1][c].dofs.end());
        std::vector<int> cp = sepCenters(e, ell);
        s.ncenter = (int)cp.size();
        s.dofs.insert(s.dofs.end(), cp.begin(), cp.end());
      }
    }
    for (int b = 0; b < nboxAt(ell); b++) {
      BoxSym& box = B_[ell][b];
      box.selfkids = selfChildren(b, ell);
      for (int c : box.selfkids)
        box.piv.insert(box.piv.end(), S_[ell + 1][c].dofs.begin(), S_[ell + 1][c].dofs.end());
      std::vector<int> cp = boxCenters(b, ell);
      box.ncenter = (int)cp.size();
      box.piv.insert(box.piv.end(), cp.begin(), cp.end());
      box.nbseps = nborSeps(b, ell);
      for (int e : box.nbseps) {
        box.bdoff.push_back(e == -1 ? -1 : (int)box.bd.size());
        if (e != -1) box.bd.insert(box.bd.end(), S_[ell][e].dofs.begin(), S_[ell][e].dofs.end());
      }
    }
  }
}

void Schedule::layout() {
  lv.resize(levels);
  int nf = 0, ns = 0;
  for (int ell = 0; ell < levels; ell++) {
    lv[ell].nbox = nboxAt(ell);
    lv[ell].nsep = ell >= 1 ? nsepAt(ell) : 0;
    lv[ell].front0 = nf;
    lv[ell].sep0 = ns;
    nf += lv[ell].nbox;
    ns += lv[ell].nsep;
  }
  fronts.resize(nf);
  seps.resize(ns);
  int64_t off = 0, doff = 0;
  for (int ell = 0; ell < levels; ell++) {
    for (int b = 0; b < lv[ell].nbox; b++) {
      BoxSym& bx = B_[ell][b];
      Front& f = fronts[lv[ell].front0 + b];
      f.level = ell;
      f.box = b;
      f.n = (int)bx.piv.size();
      f.m = (int)bx.bd.size();
      f.N = f.n + f.m;
      f.ld = (int)roundUp(f.N, 8);
      f.off = off;
      off += roundUp((int64_t)f.ld * f.N, 32);
      f.dof_off = doff;
      dofs.insert(dofs.end(), bx.piv.begin(), bx.piv.end());
      dofs.insert(dofs.end(), bx.bd.begin(), bx.bd.end());
      doff += f.N;
      if (ell == 0) {
        f.parent = -1;
      } else {
        int bps = 1 << ell, x = b % bps, y = (b / bps) % bps, z = dim == 3 ? b / (bps * bps) : 0;
        int pb = 1 << (ell - 1);
        int p = (x / 2) + (y / 2) * pb + (dim == 3 ? (z / 2) * pb * pb : 0);
        f.parent = lv[ell - 1].front0 + p;
      }
    }
  }
  front_elems = off;
  int64_t soff = 0;
  for (int ell = 1; ell < levels; ell++) {
    for (int e = 0; e < lv[ell].nsep; e++) {
      SepSym& sy = S_[ell][e];
      Sep& s = seps[lv[ell].sep0 + e];
      s.level = ell;
      s.idx = e;
      s.s = (int)sy.dofs.size();
      s.ld = (int)roundUp(std::max(s.s, 1), 8);
      s.off = soff;
      soff += roundUp((int64_t)s.ld * s.s, 32);
      s.dof_off = doff;
      dofs.insert(dofs.end(), sy.dofs.begin(), sy.dofs.end());
      doff += s.s;
      int nbx[2];
      nborBoxes(e, ell, nbx);
      for (int k = 0; k < 2; k++) {
        const BoxSym& bx = B_[ell][nbx[k]];
        int pos = -1;
        for (size_t q = 0; q < bx.nbseps.size(); q++)
          if (bx.nbseps[q] == e) pos = bx.bdoff[q];
        if (pos < 0) throw std::logic_error("separator not in its box's boundary");
        s.box[k] = lv[ell].front0 + nbx[k];
        s.bdpos[k] = (int)bx.piv.size() + pos;
      }
    }
  }
  sep_elems = soff;
}

namespace {
enum SegKind { SG_PIV = 0, SG_LSEP, SG_CSEP, SG_BCENTER, SG_ECENTER };
struct Seg {
  int kind, id, pos, len, parent;  // parent: level-ell separator of a boundary segment
  bool piv;
};
}  // namespace

void Schedule::buildTasks() {
  front_task_ptr.assign(fronts.size() + 1, 0);
  sep_task_ptr.assign(seps.size() + 1, 0);
  auto mk = [](int kind, int16_t dar, int64_t doff, int dld, int rows, int cols) {
    Task t;
    t.dst_off = doff;
    t.src_off = 0;
    t.dst_ld = dld;
    t.src_ld = 0;
    t.rows = rows;
    t.cols = cols;
    t.kind = kind;
    t.dst_arena = dar;
    t.src_arena = AR_FRONT;
    t.row_dof = t.col_dof = 0;
    t.trans = 0;
    t.lower = 0;
    t.owner = 0;
    return t;
  };
  for (size_t fi = 0; fi < fronts.size(); fi++) {
    const Front& F = fronts[fi];
    const int ell = F.level, b = F.box;
    const BoxSym& bx = B_[ell][b];
    std::vector<Seg> segs;
    if (ell == levels - 1) {
      segs.push_back({SG_PIV, -1, 0, F.n, -1, true});
      for (size_t q = 0; q < bx.nbseps.size(); q++) {
        int e = bx.nbseps[q];
        if (e == -1) continue;
        segs.push_back({SG_LSEP, e, F.n + bx.bdoff[q], (int)S_[ell][e].dofs.size(), e, false});
      }
    } else {
      int pos = 0;
      for (int c : bx.selfkids) {
        int len = (int)S_[ell + 1][c].dofs.size();
        segs.push_back({SG_CSEP, c, pos, len, -1, true});
        pos += len;
      }
      if (bx.ncenter) segs.push_back({SG_BCENTER, -1, pos, bx.ncenter, -1, true});
      for (size_t q = 0; q < bx.nbseps.size(); q++) {
        int E = bx.nbseps[q];
        if (E == -1) continue;
        int p = F.n + bx.bdoff[q];
        for (int c : S_[ell][E].kids) {
          int len = (int)S_[ell + 1][c].dofs.size();
          segs.push_back({SG_CSEP, c, p, len, E, false});
          p += len;
        }
        if (S_[ell][E].ncenter) segs.push_back({SG_ECENTER, -1, p, S_[ell][E].ncenter, E, false});
      }
    }
    std::vector<int> kids = ell < levels - 1 ? childBoxes(b, ell) : std::vector<int>();
    auto childBlock = [&](int s, int t, int rowpos, int colpos, int rows, int cols) -> bool {
      // a child box whose boundary holds both separators s and t (level ell+1)
      for (int c : kids) {
        const BoxSym& cb = B_[ell + 1][c];
        int os = -1, ot = -1;
        for (size_t q = 0; q < cb.nbseps.size(); q++) {
          if (cb.nbseps[q] == s) os = cb.bdoff[q];
          if (cb.nbseps[q] == t) ot = cb.bdoff[q];
        }
        if (os < 0 || ot < 0) continue;
        const Front& C = fronts[lv[ell + 1].front0 + c];
        Task tk = mk(TK_COPY, AR_FRONT, F.off + rowpos + (int64_t)colpos * F.ld, F.ld, rows, cols);
        tk.src_arena = AR_FRONT;
        tk.src_ld = C.ld;
        if (os > ot || full_storage) {   // the child holds block (s, t) itself
          tk.src_off = C.off + (C.n + os) + (int64_t)(C.n + ot) * C.ld;
        } else {
          tk.trans = 1;
          tk.src_off = C.off + (C.n + ot) + (int64_t)(C.n + os) * C.ld;
        }
        tk.owner = (int)fi;
        front_tasks.push_back(tk);
        return true;
      }
      return false;
    };
    for (size_t a = 0; a < segs.size(); a++) {
      for (size_t bb = 0; bb < (full_storage ? segs.size() : a + 1); bb++) {
        const Seg& R = segs[a];
        const Seg& C = segs[bb];
        const int64_t doff = F.off + R.pos + (int64_t)C.pos * F.ld;
        Task t = mk(TK_ZERO, AR_FRONT, doff, F.ld, R.len, C.len);
        t.owner = (int)fi;
        t.lower = (a == bb && !full_storage) ? 1 : 0;
        auto sparse = [&]() {
          t.kind = TK_SPARSE;
          t.row_dof = (int32_t)(F.dof_off + R.pos);
          t.col_dof = (int32_t)(F.dof_off + C.pos);
        };
        if (ell == levels - 1) {
          // leaf front: everything from the sparse matrix, except the diagonal
          // blocks of boundary separators, which start at zero so that the
          // trailing block ends up holding the Schur complement alone there.
          if (a == bb && !R.piv) t.kind = TK_ZERO;
          else sparse();
          front_tasks.push_back(t);
          continue;
        }
        if (a == bb) {
          if (R.kind == SG_CSEP && R.piv) {
            const Sep& S = seps[lv[ell + 1].sep0 + R.id];
            t.kind = TK_COPY;
            t.src_arena = AR_SEP;
            t.src_off = S.off;
            t.src_ld = S.ld;
          } else if (R.kind == SG_BCENTER) {
            sparse();
          }  // boundary diagonal blocks: zero
          front_tasks.push_back(t);
          continue;
        }
        if (R.piv && C.piv) {                       // A22 off-diagonal block
          if (R.kind == SG_BCENTER || C.kind == SG_BCENTER) {
            sparse();
          } else if (childBlock(R.id, C.id, R.pos, C.pos, R.len, C.len)) {
            continue;
          }
        } else if (!R.piv && C.piv) {               // A12
          if (R.kind == SG_ECENTER) {
            sparse();
          } else if (C.kind == SG_CSEP && childBlock(R.id, C.id, R.pos, C.pos, R.len, C.len)) {
            continue;
          }
        } else if (R.piv && !C.piv) {               // A21 (full storage only): A12's mirror
          if (C.kind == SG_ECENTER) {
            sparse();
          } else if (R.kind == SG_CSEP && childBlock(R.id, C.id, R.pos, C.pos, R.len, C.len)) {
            continue;
          }
        } else {                                    // A11 (boundary x boundary)
          if (R.parent != C.parent && R.kind == SG_CSEP && C.kind == SG_CSEP &&
              childBlock(R.id, C.id, R.pos, C.pos, R.len, C.len))
            continue;
        }
        front_tasks.push_back(t);
      }
    }
    front_task_ptr[fi + 1] = (int64_t)front_tasks.size();
  }

  // separators: base assembly (mf2d.cpp:591-595 leaf, 274-319 upper)
  for (size_t si = 0; si < seps.size(); si++) {
    const Sep& S = seps[si];
    const int ell = S.level;
    auto base = [&](int kind, int rpos, int cpos, int rows, int cols, int lower) {
      Task t = mk(kind, AR_SEP, S.off + rpos + (int64_t)cpos * S.ld, S.ld, rows, cols);
      t.lower = lower;
      t.owner = (int)si;
      t.row_dof = (int32_t)(S.dof_off + rpos);
      t.col_dof = (int32_t)(S.dof_off + cpos);
      return t;
    };
    if (ell == levels - 1) {
      sep_tasks.push_back(base(TK_SPARSE, 0, 0, S.s, S.s, full_storage ? 0 : 1));
    } else {
      const SepSym& sy = S_[ell][S.idx];
      struct P { int pos, len, kid; };
      std::vector<P> parts;
      int pos = 0;
      for (int c : sy.kids) {
        int len = (int)S_[ell + 1][c].dofs.size();
        parts.push_back({pos, len, c});
        pos += len;
      }
      if (sy.ncenter) parts.push_back({pos, sy.ncenter, -1});
      for (size_t a = 0; a < parts.size(); a++)
        for (size_t bb = 0; bb < (full_storage ? parts.size() : a + 1); bb++) {
          const P& R = parts[a];
          const P& C = parts[bb];
          if (R.kid < 0 || C.kid < 0) {
            sep_tasks.push_back(base(TK_SPARSE, R.pos, C.pos, R.len, C.len, a == bb && !full_storage));
          } else if (a == bb) {
            const Sep& K = seps[lv[ell + 1].sep0 + R.kid];
            Task t = base(TK_COPY, R.pos, R.pos, R.len, R.len, full_storage ? 0 : 1);
            t.src_arena = AR_SEP;
            t.src_off = K.off;
            t.src_ld = K.ld;
            sep_tasks.push_back(t);
          } else {
            sep_tasks.push_back(base(TK_ZERO, R.pos, C.pos, R.len, C.len, 0));
          }
        }
    }
    sep_task_ptr[si + 1] = (int64_t)sep_tasks.size();
    // accumulation (ScatterAdd_, mf2d.cpp:599-606): two adds, box order
    for (int k = 0; k < 2; k++) {
      const Front& F = fronts[S.box[k]];
      Task t = mk(TK_ADD, AR_SEP, S.off, S.ld, S.s, S.s);
      t.lower = full_storage ? 0 : 1;
      t.src_arena = AR_FRONT;
      t.src_off = F.off + S.bdpos[k] + (int64_t)S.bdpos[k] * F.ld;
      t.src_ld = F.ld;
      t.owner = (int)si;
      sep_add_tasks.push_back(t);
    }
  }
}

Schedule::Schedule(std::vector<Schedule>&& batch) {
  if (batch.empty()) throw std::invalid_argument("empty batch");
  parts = std::move(batch);
  const int P = (int)parts.size();
  const Schedule& p0 = parts[0];
  dim = p0.dim;
  width = p0.width;
  for (int a = 0; a < 3; a++) {
    N[a] = p0.N[a];
    bw[a] = p0.bw[a];
  }
  levels = 0;
  for (const Schedule& q : parts) levels = std::max(levels, q.levels);
  auto shift = [&](int p) { return levels - parts[p].levels; };
  dof_base.assign(P + 1, 0);
  std::vector<int64_t> fbase(P + 1, 0), sbase(P + 1, 0), tbase(P + 1, 0);
  for (int p = 0; p < P; p++) {
    dof_base[p + 1] = dof_base[p] + parts[p].ndof;
    fbase[p + 1] = fbase[p] + parts[p].front_elems;
    sbase[p + 1] = sbase[p] + parts[p].sep_elems;
    tbase[p + 1] = tbase[p] + (int64_t)parts[p].dofs.size();
  }
  ndof = dof_base[P];
  if (ndof > 0x7fffffffLL) throw std::invalid_argument("more than 2^31-1 DOFs in the batch");
  if (tbase[P] > 0x7fffffffLL) throw std::invalid_argument("DOF table too large for the batch");
  front_elems = fbase[P];
  sep_elems = sbase[P];
  // levels and renumbering: level by level, part by part, local order inside
  lv.assign(levels, LevelInfo{0, 0, 0, 0});
  for (int ml = 0; ml < levels; ml++)
    for (int p = 0; p < P; p++) {
      const int pl = ml - shift(p);
      if (pl < 0) continue;
      lv[ml].nbox += parts[p].lv[pl].nbox;
      lv[ml].nsep += parts[p].lv[pl].nsep;
    }
  int nf = 0, ns = 0;
  for (int ml = 0; ml < levels; ml++) {
    lv[ml].front0 = nf;
    lv[ml].sep0 = ns;
    nf += lv[ml].nbox;
    ns += lv[ml].nsep;
  }
  front_map.resize(P);
  sep_map.resize(P);
  std::vector<std::pair<int, int>> fsrc(nf), ssrc(ns);   // id here -> (part, local id)
  for (int p = 0; p < P; p++) {
    front_map[p].assign(parts[p].fronts.size(), -1);
    sep_map[p].assign(parts[p].seps.size(), -1);
  }
  for (int ml = 0; ml < levels; ml++) {
    int fc = lv[ml].front0, sc = lv[ml].sep0;
    for (int p = 0; p < P; p++) {
      const int pl = ml - shift(p);
      if (pl < 0) continue;
      const LevelInfo& L = parts[p].lv[pl];
      for (int b = 0; b < L.nbox; b++) {
        front_map[p][L.front0 + b] = fc;
        fsrc[fc++] = {p, L.front0 + b};
      }
      for (int e = 0; e < L.nsep; e++) {
        sep_map[p][L.sep0 + e] = sc;
        ssrc[sc++] = {p, L.sep0 + e};
      }
    }
  }
  fronts.resize(nf);
  seps.resize(ns);
  dofs.reserve((size_t)tbase[P]);
  // per part: (old table offset, new table offset, length), sorted by old offset
  std::vector<std::vector<std::array<int64_t, 3>>> tmap(P);
  for (int i = 0; i < nf; i++) {
    const int p = fsrc[i].first;
    Front f = parts[p].fronts[fsrc[i].second];
    tmap[p].push_back({f.dof_off, (int64_t)dofs.size(), f.N});
    for (int k = 0; k < f.N; k++)
      dofs.push_back((int32_t)(parts[p].dofs[f.dof_off + k] + dof_base[p]));
    f.level += shift(p);
    f.off += fbase[p];
    f.dof_off = tmap[p].back()[1];
    f.parent = f.parent >= 0 ? front_map[p][f.parent] : -1;
    fronts[i] = f;
  }
  for (int i = 0; i < ns; i++) {
    const int p = ssrc[i].first;
    Sep q = parts[p].seps[ssrc[i].second];
    tmap[p].push_back({q.dof_off, (int64_t)dofs.size(), q.s});
    for (int k = 0; k < q.s; k++)
      dofs.push_back((int32_t)(parts[p].dofs[q.dof_off + k] + dof_base[p]));
    q.level += shift(p);
    q.off += sbase[p];
    q.dof_off = tmap[p].back()[1];
    q.box[0] = front_map[p][q.box[0]];
    q.box[1] = front_map[p][q.box[1]];
    seps[i] = q;
  }
  for (auto& m : tmap) std::sort(m.begin(), m.end());
  auto tpos = [&](int p, int64_t old) -> int32_t {   // old table index of part p -> new
    const auto& m = tmap[p];
    auto it = std::upper_bound(m.begin(), m.end(),
                               std::array<int64_t, 3>{old, INT64_MAX, INT64_MAX});
    if (it == m.begin()) throw std::logic_error("DOF table index outside every list");
    --it;
    if (old >= (*it)[0] + std::max<int64_t>((*it)[2], 1))
      throw std::logic_error("DOF table index outside every list");
    return (int32_t)((*it)[1] + (old - (*it)[0]));
  };
  auto remap = [&](Task t, int p, bool front_owner) {
    t.dst_off += t.dst_arena == AR_FRONT ? fbase[p] : sbase[p];
    if (t.kind != TK_SPARSE) t.src_off += t.src_arena == AR_FRONT ? fbase[p] : sbase[p];
    if (t.kind == TK_SPARSE) {
      t.row_dof = t.rows > 0 ? tpos(p, t.row_dof) : 0;
      t.col_dof = t.cols > 0 ? tpos(p, t.col_dof) : 0;
    }
    t.owner = front_owner ? front_map[p][t.owner] : sep_map[p][t.owner];
    return t;
  };
  front_task_ptr.assign(nf + 1, 0);
  for (int i = 0; i < nf; i++) {
    const Schedule& q = parts[fsrc[i].first];
    const int lf = fsrc[i].second;
    for (int64_t k = q.front_task_ptr[lf]; k < q.front_task_ptr[lf + 1]; k++)
      front_tasks.push_back(remap(q.front_tasks[k], fsrc[i].first, true));
    front_task_ptr[i + 1] = (int64_t)front_tasks.size();
  }
  sep_task_ptr.assign(ns + 1, 0);
  for (int i = 0; i < ns; i++) {
    const Schedule& q = parts[ssrc[i].first];
    const int ls = ssrc[i].second;
    for (int64_t k = q.sep_task_ptr[ls]; k < q.sep_task_ptr[ls + 1]; k++)
      sep_tasks.push_back(remap(q.sep_tasks[k], ssrc[i].first, false));
    sep_task_ptr[i + 1] = (int64_t)sep_tasks.size();
    for (int k = 0; k < 2; k++)
      sep_add_tasks.push_back(remap(q.sep_add_tasks[2 * (size_t)ls + k], ssrc[i].first, false));
  }
}

int Schedule::leaf_of_dof(int dof) const {
  if (forest()) {
    const int p = (int)(std::upper_bound(dof_base.begin(), dof_base.end(), (int64_t)dof) -
                        dof_base.begin()) - 1;
    return front_map[p][parts[p].leaf_of_dof((int)(dof - dof_base[p]))];
  }
  int bps = 1 << (levels - 1);
  int c[3];
  int64_t d = dof;
  c[0] = (int)(d % N[0]);
  d /= N[0];
  c[1] = (int)(d % N[1]);
  c[2] = (int)(d / N[1]);
  int box = 0, mul = 1;
  for (int a = 0; a < dim; a++) {
    // i / (b + w) as mf2d.cpp:169-170; the last box absorbs the remainder
    int q = std::min(c[a] / (bw[a] + width), bps - 1);
    box += q * mul;
    mul *= bps;
  }
  return lv[levels - 1].front0 + box;
}

// The reference marks the leaf of each modified DOF (mf2d.cpp:163-174) and, at
// every level, the parents of both boxes next to each marked separator
// (mf2d.cpp:607-614).  A box's Schur complement depends only on its own subtree
// and a separator is recomputed whenever a box next to it is, so refactoring
// the root paths of the marked leaves gives the same factors with fewer fronts.
size_t Schedule::dirty_fronts(const int* mod, int nmod, std::vector<char>& dirty) const {
  dirty.assign(fronts.size(), 0);
  size_t nd = 0;
  if (forest()) {
    // each touched problem refactors its own root paths (and its root)
    std::vector<std::vector<int>> local(parts.size());
    for (int i = 0; i < nmod; i++) {
      const int p = (int)(std::upper_bound(dof_base.begin(), dof_base.end(), (int64_t)mod[i]) -
                          dof_base.begin()) - 1;
      local[p].push_back((int)(mod[i] - dof_base[p]));
    }
    for (size_t p = 0; p < parts.size(); p++) {
      if (local[p].empty()) continue;
      std::vector<char> d;
      parts[p].dirty_fronts(local[p].data(), (int)local[p].size(), d);
      for (size_t f = 0; f < d.size(); f++)
        if (d[f]) {
          dirty[front_map[p][f]] = 1;
          nd++;
        }
    }
    return nd;
  }
  for (int i = 0; i < nmod; i++) {
    int f = leaf_of_dof(mod[i]);
    while (f >= 0 && !dirty[f]) {
      dirty[f] = 1;
      nd++;
      f = fronts[f].parent;
    }
  }
  if (!dirty[0]) {
    dirty[0] = 1;   // the root is always refactored (mf2d.cpp:633-657)
    nd++;
  }
  return nd;
}

double Schedule::front_flops(const Front& f) const {
  double n = f.n, m = f.m;
  return n * n * n / 3.0 + n * n * m + n * m * m;
}

double Schedule::total_flops() const {
  double s = 0;
  for (const Front& f : fronts) s += front_flops(f);
  return s;
}

}  // namespace mfgpu
