// Symbolic elimination-tree schedule of the box/separator multifrontal method.
//
// Restates the reference's symbolic setup (src/DE/mf2d.cpp:8-148 and 186-446,
// src/DE/mf3d.cpp:26-206 and 253-702, tree topology src/DE/tree2d_common.cpp,
// src/DE/tree3d_common.cpp) on the host, once per problem, and flattens it into
// the tables the device kernels read:
//   * per front (one per box): pivot and boundary DOF lists in the reference's
//     exact order, sizes and offsets into the factor arena;
//   * per separator (edge in 2D, face in 3D): DOF list and arena offset;
//   * block-copy "assembly tasks" that build every front and every separator
//     from its sources (children's update matrices, child separators, the
//     sparse matrix) with the reference's replace / add semantics.
// Nothing here touches the GPU; the handle uploads the tables.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mfgpu {

// Kinds of assembly task.
enum TaskKind : int32_t {
  TK_ZERO = 0,    // dst = 0
  TK_COPY = 1,    // dst = src            (src in the front arena or sep arena)
  TK_SPARSE = 2,  // dst = A(row dof, col dof) gathered from the CSR matrix
  TK_ADD = 3      // dst += src
};
enum Arena : int32_t { AR_FRONT = 0, AR_SEP = 1 };

// One rectangular block operation.  Element (i, j), 0 <= i < rows, 0 <= j < cols:
//   dst[dst_off + i + j*dst_ld]  (op)  src[src_off + (trans ? j + i*src_ld : i + j*src_ld)]
// lower != 0 restricts the block to i >= j (diagonal blocks of symmetric storage).
// For TK_SPARSE the DOFs are dofs[row_dof + i] and dofs[col_dof + j], and
// src_off is the element offset of the matrix's CSR values (0 here; the
// serving loop sets it when one plan covers several matrices).
struct Task {
  int64_t dst_off;
  int64_t src_off;
  int32_t dst_ld, src_ld;
  int32_t rows, cols;
  int32_t kind;
  int16_t dst_arena, src_arena;
  int32_t row_dof, col_dof;
  int16_t trans, lower;
  int32_t owner;  // front id (front tasks) or separator id (separator tasks)
};
static_assert(sizeof(Task) == 56, "task layout");

struct Front {
  int level, box;
  int n, m;           // pivots, boundary
  int N, ld;          // n + m, leading dimension (column-major, lower triangle used)
  int64_t off;        // element offset in the front arena
  int64_t dof_off;    // offset of [pivots..., boundary...] in the DOF table
  int parent;         // global front id of the parent box, -1 for the root
};

struct Sep {
  int level, idx;
  int s, ld;
  int64_t off;        // element offset in the separator arena
  int64_t dof_off;    // offset of the DOF list in the DOF table
  int box[2];         // global front ids of the two adjacent boxes, reference order
  int bdpos[2];       // row of this separator inside each box's front (n + offset)
};

struct LevelInfo {
  int nbox, nsep;
  int front0, sep0;   // first global front / separator id of this level
};

class Schedule {
 public:
  // Throws std::runtime_error with the reference's messages on bad parameters.
  // full_storage: task tables for nonsymmetric matrices (every block of every
  // front and separator, both triangles); by default the tables fill the lower
  // triangles only, which is all the Cholesky kernels read.
  Schedule(int dim, int nx, int ny, int nz, int width, int max_side, bool full_storage = false);

  // A batch of independent problems as one forest over their block-diagonal
  // matrix.  Levels are aligned at the leaves: part p's level l is level
  // l + (levels - parts[p].levels) here, so one launch per level covers the
  // fronts of every problem at that height.  Fronts and separators are
  // renumbered level by level (part by part inside a level), DOFs of part p
  // are shifted by dof_base[p], arena offsets by the parts' arena sizes, and
  // the DOF table keeps the single-problem layout (all fronts, then all
  // separators).
  explicit Schedule(std::vector<Schedule>&& batch);

  std::vector<Schedule> parts;        // the batch members (empty for one problem)
  std::vector<int64_t> dof_base;      // parts.size() + 1 DOF offsets
  std::vector<std::vector<int>> front_map, sep_map;   // part-local id -> id here
  bool forest() const { return !parts.empty(); }

  int dim, N[3], width, levels;
  bool full_storage = false;   // tables fill both triangles (nonsymmetric matrices)
  int bw[3];                        // leaf box widths
  int64_t ndof;
  std::vector<LevelInfo> lv;        // index = level (0 = root)
  std::vector<Front> fronts;        // global front ids: level by level, root first
  std::vector<Sep> seps;            // global separator ids: level 1..L-1
  std::vector<int32_t> dofs;        // DOF table (fronts, then separators)
  int64_t front_elems = 0, sep_elems = 0;

  // Assembly tasks, grouped per owner so subsets can be selected for updates.
  std::vector<Task> front_tasks;          // ordered by front id
  std::vector<int64_t> front_task_ptr;    // size fronts+1
  std::vector<Task> sep_tasks;            // base assembly of separators
  std::vector<int64_t> sep_task_ptr;      // size seps+1
  std::vector<Task> sep_add_tasks;        // two per separator: += box0 block, += box1 block
  // Per leaf box the global front id, for the modified-DOF -> leaf map.
  int leaf_of_dof(int dof) const;
  // Fronts a localized update must refactor: the leaves holding modified DOFs
  // and all their ancestors, plus the root.  Returns how many are marked.
  size_t dirty_fronts(const int* mod, int nmod, std::vector<char>& dirty) const;

  // Work model (Cholesky form): sum over fronts of n^3/3 + n^2 m + n m^2.
  double front_flops(const Front& f) const;
  double total_flops() const;

  int front_id(int level, int box) const { return lv[level].front0 + box; }
  int sep_id(int level, int e) const { return lv[level].sep0 + e; }

 private:
  // per level scratch used while building (kept small)
  struct BoxSym {
    std::vector<int> piv, bd;
    std::vector<int> nbseps;      // nbor separators incl. -1, reference order
    std::vector<int> bdoff;       // offset of each nbor separator in bd (-1 if absent)
    std::vector<int> selfkids;    // self child separators (level+1), sorted
    int ncenter = 0;
  };
  struct SepSym {
    std::vector<int> dofs;
    std::vector<int> kids;        // child separators (level+1)
    int ncenter = 0;
  };
  std::vector<std::vector<BoxSym>> B_;
  std::vector<std::vector<SepSym>> S_;

  // topology helpers
  std::vector<int> nborSeps(int b, int ell) const;
  void nborBoxes(int e, int ell, int out[2]) const;
  std::vector<int> childSeps(int e, int ell) const;
  std::vector<int> childBoxes(int b, int ell) const;
  std::vector<int> selfChildren(int b, int ell) const;
  int nsepAt(int ell) const;
  int nboxAt(int ell) const;
  int bwidth(int ell, int axis, bool below) const;
  std::vector<int> boxCenters(int b, int ell) const;
  std::vector<int> sepCenters(int e, int ell) const;
  void block(const int lo[3], const int hi[3], std::vector<int>& out) const;

  void buildLeaves();
  void buildUpper();
  void layout();
  void buildTasks();
};

}  // namespace mfgpu
